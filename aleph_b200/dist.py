"""Amplitude sharding: one state vector over 2^g ranks, one or more per GPU.

The layout follows the reference's distributed state (crates/aleph-ir/src/dist,
crates/aleph-cuda/src/dist): physical qubits 0..m-1 are local (m = n - g), the
top g are global, and rank r holds the 2^m amplitudes whose global bits spell
r. The plan is a list of local steps and exchanges:

* A local step is a stretch of the circuit in which every gate acts
  non-diagonally on local qubits only. Each rank runs it as ONE
  gate stream on its own slice through the engine (planned and fused like
  any in-core run), after per-rank specialisation (``specialize``): a
  control on a global qubit keeps or drops the gate for the whole rank, and
  a diagonal gate or DiagonalPhase term on global qubits becomes a smaller
  diagonal (or a phase) on the local ones.
* An exchange swaps one global qubit with the top local qubit m-1. Rank r
  and its partner r ^ (1 << j) swap the half of their slices whose top local
  bit differs from bit j of the rank: one contiguous 2^(m-1)-amplitude
  region each way, moved in chunks over NCCL (NVLink between GPUs) or by a
  device copy when both ranks live on the same GPU (``Exchange``), like the
  reference's chunk-pair transfers (crates/aleph-cuda/src/dist/exchange.rs,
  nccl.rs:212-237).

The router (``plan_dist``) brings a global qubit local just before a gate
needs it non-diagonally, evicting the local qubit whose next non-diagonal use
lies furthest ahead (Belady's rule; the reference's routers live in
crates/aleph-ir/src/dist/plan.rs). An evicted qubit that is not already at
position m-1 is first moved there by a SWAP inside the local step, which the
engine applies as a qubit relabel plus one permutation pass. ``final_map``
gives each logical qubit's physical position at the end.
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import abi
from . import circuit as C

# gates whose first qubit is a control and act non-diagonally on the rest
_CONTROL_FIRST = {"Cnot": 1, "CRx": 1, "CRy": 1, "Toffoli": 2}


class DistError(ValueError):
    """A circuit or layout the distributed path does not support."""


@dataclass(frozen=True)
class DistLayout:
    """n qubits over 2^g ranks of 2^(n-g) amplitudes (DistLayout,
    crates/aleph-ir/src/dist/mod.rs)."""

    n: int
    g: int

    def __post_init__(self):
        if self.g < 0 or self.n - self.g < 1 or self.n > 64:
            raise DistError(f"layout needs 0 <= g < n <= 64 (n={self.n}, g={self.g})")

    @property
    def m(self) -> int:
        return self.n - self.g

    @property
    def ranks(self) -> int:
        return 1 << self.g

    def is_global(self, p: int) -> bool:
        return p >= self.m

    def rank_bit(self, rank: int, p: int) -> int:
        return (rank >> (p - self.m)) & 1


@dataclass
class LocalStep:
    instructions: list  # physical qubit indices


@dataclass
class ExchangeStep:
    global_qubit: int  # physical position >= m, swapped with position m-1


@dataclass
class DistPlan:
    layout: DistLayout
    steps: list
    final_map: list  # logical qubit -> physical position

    def exchanges(self) -> int:
        return sum(isinstance(s, ExchangeStep) for s in self.steps)


# ---- routing -------------------------------------------------------------------------------
def nondiagonal_targets(inst) -> tuple:
    """The qubits an instruction acts on non-diagonally (those must be local
    when it runs). Controls never need to be: they specialise per rank."""
    if isinstance(inst, (C.DiagonalPhase, C.Barrier)):
        return ()
    if isinstance(inst, (C.Measure, C.Reset)) or not isinstance(inst, C.GateInstance):
        raise DistError(f"{type(inst).__name__} is not supported by the distributed path")
    g = inst.gate
    if g.is_diagonal():
        return ()
    skip = _CONTROL_FIRST.get(g.name, 0)
    return inst.qubits[skip:]


def _remap(inst, phys):
    if isinstance(inst, C.GateInstance):
        return C.GateInstance(inst.gate, [phys[q] for q in inst.qubits], [phys[c] for c in inst.controls])
    if isinstance(inst, C.DiagonalPhase):
        def mp(mask):
            out = 0
            for q in range(inst.n_qubits):
                if (mask >> q) & 1:
                    out |= 1 << phys[q]
            return out
        return C.DiagonalPhase(inst.n_qubits, [C.PhaseTerm(tuple(mp(c) for c in t.conds), t.angle)
                                               for t in inst.terms])
    return inst


def plan_dist(instructions: Sequence, layout: DistLayout) -> DistPlan:
    """Local steps and exchanges for ``instructions`` (logical qubits) on
    ``layout``; every instruction of a local step names physical qubits."""
    n, m = layout.n, layout.m
    insts = list(instructions)
    for inst in insts:
        for q in (inst.qubits + inst.controls if isinstance(inst, C.GateInstance) else ()):
            if q >= n:
                raise DistError(f"qubit {q} out of range for {n} qubits")
    # next non-diagonal use of each logical qubit, for Belady eviction
    uses: list[list[int]] = [[] for _ in range(n)]
    for i, inst in enumerate(insts):
        for q in nondiagonal_targets(inst):
            uses[q].append(i)
    ptr = [0] * n

    def next_use(q: int, i: int) -> int:
        u = uses[q]
        while ptr[q] < len(u) and u[ptr[q]] <= i:
            ptr[q] += 1
        return u[ptr[q]] if ptr[q] < len(u) else len(insts) + 1

    phys = list(range(n))  # logical -> physical
    logi = list(range(n))  # physical -> logical
    steps: list = []
    cur: list = []

    def swap_positions(a: int, b: int):
        la, lb = logi[a], logi[b]
        logi[a], logi[b] = lb, la
        phys[la], phys[lb] = b, a

    for i, inst in enumerate(insts):
        targets = nondiagonal_targets(inst)
        for q in targets:
            if phys[q] < m:
                continue
            busy = {phys[t] for t in targets if phys[t] < m}
            cands = [p for p in range(m) if p not in busy]
            if not cands:
                raise DistError(f"a gate on {len(targets)} qubits needs more than {m} local qubits")
            victim = max(cands, key=lambda p: (next_use(logi[p], i), p == m - 1))
            if victim != m - 1:
                cur.append(C.GateInstance(C.Swap(), [victim, m - 1]))
                swap_positions(victim, m - 1)
            if cur:
                steps.append(LocalStep(cur))
                cur = []
            steps.append(ExchangeStep(phys[q]))
            swap_positions(phys[q], m - 1)
        cur.append(_remap(inst, phys))
    if cur:
        steps.append(LocalStep(cur))
    return DistPlan(layout, steps, list(phys))


# ---- per-rank specialisation --------------------------------------------------------------
def _gate_matrix(g: C.Gate, nq: int) -> np.ndarray:
    """Gate::matrix through the engine's own (aleph_b200_gate_matrix)."""
    inst = C.GateInstance(g, list(range(nq)))
    flat = C.flatten([inst])
    out = (ct.c_double * 128)()
    dim = ct.c_int()
    L = abi.load_library()
    st = L.aleph_b200_gate_matrix(flat.instrs, flat.matrix_ptr, flat.matrix.size // 2, out, ct.byref(dim))
    if st != abi.OK:
        raise DistError(f"{g.name}: no matrix ({abi.STATUS_NAMES.get(st, st)})")
    d = dim.value
    a = np.frombuffer(out, dtype=np.float64)[: 2 * d * d]
    return (a[0::2] + 1j * a[1::2]).reshape(d, d)


def _phase_gate(phi: float, controls: list, m: int) -> list:
    """exp(i phi) on the states where every local control is 1 (on the whole
    slice when there is none)."""
    if phi == 0.0:
        return []
    if not controls:
        return [C.DiagonalPhase(m, [C.PhaseTerm((), float(phi))])]
    return [C.GateInstance(C.Unitary1qDiag([1.0, np.exp(1j * phi)]), [controls[-1]], controls[:-1])]


def specialize(inst, layout: DistLayout, rank: int) -> list:
    """Rank ``rank``'s local instructions for one physical instruction
    (specialize, crates/aleph-ir/src/dist/specialize.rs): qubits < m stay,
    global qubits are fixed to the rank's bits."""
    m = layout.m
    if isinstance(inst, C.Barrier):
        return []
    if isinstance(inst, C.DiagonalPhase):
        return _specialize_phase(inst, layout, rank)
    g = inst.gate
    controls = []
    for c in inst.controls:
        if layout.is_global(c):
            if layout.rank_bit(rank, c) == 0:
                return []
        else:
            controls.append(c)
    qs = list(inst.qubits)
    if not any(layout.is_global(q) for q in qs):
        return [C.GateInstance(g, qs, controls)]
    skip = _CONTROL_FIRST.get(g.name, 0)
    if skip and not g.is_diagonal():
        kept = []
        for c in qs[:skip]:
            if layout.is_global(c):
                if layout.rank_bit(rank, c) == 0:
                    return []
            else:
                kept.append(c)
        rest = qs[skip:]
        if any(layout.is_global(q) for q in rest):
            raise DistError(f"{g.name} on a global target reached a local step")
        if g.name == "Toffoli":
            reduced = C.Cnot() if len(kept) == 1 else C.X()
            return [C.GateInstance(reduced, kept + rest, controls)]
        reduced = {"Cnot": C.X(), "CRx": C.Rx(g.params[0] if g.params else 0.0),
                   "CRy": C.Ry(g.params[0] if g.params else 0.0)}[g.name]
        return [C.GateInstance(reduced, rest, controls)]
    if not g.is_diagonal():
        raise DistError(f"{g.name} on a global qubit reached a local step")
    # a diagonal gate: its phase function restricted to the rank's global bits
    k = len(qs)
    d = np.diag(_gate_matrix(g, k)) if g.name not in ("Unitary1qDiag", "Unitary2qDiag") else \
        np.asarray(g.matrix, dtype=np.complex128).reshape(-1)
    loc = [j for j, q in enumerate(qs) if not layout.is_global(q)]
    fixed = 0  # matrix index bits of the global operands (operand j is bit k-1-j)
    for j, q in enumerate(qs):
        if layout.is_global(q) and layout.rank_bit(rank, q):
            fixed |= 1 << (k - 1 - j)
    sub = []
    for x in range(1 << len(loc)):
        idx = fixed
        for t, j in enumerate(loc):  # loc[t] is bit len(loc)-1-t of x (MSB-first)
            if (x >> (len(loc) - 1 - t)) & 1:
                idx |= 1 << (k - 1 - j)
        sub.append(d[idx])
    sub = np.asarray(sub, dtype=np.complex128)
    if np.all(sub == 1.0):
        return []
    if not loc:
        return _phase_gate(float(np.angle(sub[0])), controls, m)
    lq = [qs[j] for j in loc]
    gate = C.Unitary1qDiag(sub) if len(lq) == 1 else C.Unitary2qDiag(sub)
    return [C.GateInstance(gate, lq, controls)]


def _specialize_phase(dp: C.DiagonalPhase, layout: DistLayout, rank: int) -> list:
    """A DiagonalPhase on the rank's slice: a condition's global bits fold
    into a fixed parity; a condition whose global parity is odd becomes the
    complement of its local parity, expanded by inclusion-exclusion."""
    m = layout.m
    lmask = (1 << m) - 1
    terms = []
    for t in dp.terms:
        plain, neg, dead = [], [], False
        for c in t.conds:
            cl, cg = c & lmask, c >> m
            odd = bin(cg & rank).count("1") & 1
            if not odd:
                if cl == 0:
                    dead = True  # parity of nothing is even: the term never fires
                    break
                plain.append(cl)
            elif cl:
                neg.append(cl)  # fires when the local parity is even
        if dead:
            continue
        for sel in range(1 << len(neg)):
            conds = plain + [neg[j] for j in range(len(neg)) if (sel >> j) & 1]
            sign = -1.0 if bin(sel).count("1") & 1 else 1.0
            terms.append(C.PhaseTerm(tuple(conds), sign * t.angle))
    return [C.DiagonalPhase(m, terms)] if terms else []


def rank_program(instructions: Sequence, layout: DistLayout, rank: int) -> list:
    out = []
    for inst in instructions:
        out.extend(specialize(inst, layout, rank))
    return out


# ---- ranks and the exchange ---------------------------------------------------------------------
def owner(rank: int, layout: DistLayout, world: int) -> int:
    """The process holding a rank: contiguous blocks of 2^g / world ranks, so
    the top log2(world) rank bits name the process (rank_device,
    crates/aleph-cuda/src/dist/exchange.rs)."""
    return rank // (layout.ranks // world)


class EngineRanks:
    """This process's rank slices as engine states on one GPU (all 2^g ranks
    when the process runs alone; its block of them under torchrun)."""

    def __init__(self, backend, layout: DistLayout, ranks: Sequence[int]):
        import torch

        self.be, self.layout, self.ranks = backend, layout, list(ranks)
        self.states = {}
        if getattr(backend, "precision", "") == "tc32":
            # a slice's norm is not 1: no end-of-stream rescale (as for the
            # tile groups of an out-of-core run)
            backend.set_tuning("renormalize", 0)
        self._torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        backend.synchronize()
        with self.stream_ctx():
            for r in self.ranks:
                self.states[r] = backend.allocate(layout.m)  # |0...0>
                if r != 0:
                    self.bytes_view(r).zero_()  # the other ranks start empty
        backend.synchronize()

    def stream_ctx(self):
        """Torch work inside this context runs on the engine's stream, in
        order with the engine's kernels."""
        return self._torch.cuda.stream(self._torch.cuda.ExternalStream(self.be.stream_ptr(), device=self.device))

    def bytes_view(self, r: int):
        """The slice of rank r as a uint8 device tensor (no copy)."""
        ptr, nbytes = self.be.state_memory(self.states[r])
        return self._torch.as_tensor(_DeviceBytes(ptr, nbytes), device=self.device)

    def apply(self, r: int, instructions: list) -> None:
        if instructions:
            self.be.apply_stream(self.states[r], instructions)

    def statevector(self, r: int) -> np.ndarray:
        return self.be.statevector(self.states[r])

    def scale(self, r: int, factor: float) -> None:
        self.be.scale_state(self.states[r], factor)

    def renormalizes(self) -> bool:
        """TC32 slices run without the end-of-stream rescale; the run restores
        the global norm once at its end instead."""
        return getattr(self.be, "precision", "") == "tc32"

    def norm_sqr(self, r: int) -> float:
        return self.be.norm_sqr(self.states[r])

    def free(self) -> None:
        for st in self.states.values():
            st.free()
        self.states = {}


class _DeviceBytes:
    """A device allocation described by __cuda_array_interface__, so that
    torch can view it without copying."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


class Exchange:
    """Swaps a global qubit with the top local qubit: for each rank pair
    (r, r ^ (1 << j)), the half of r's slice whose top local bit is the
    complement of r's bit j trades places with the same half of the partner.
    Pairs on this process swap by device copies through a scratch chunk;
    pairs across processes send and receive the chunks over torch.distributed
    (NCCL between GPUs, gloo on CPU), all of one step in one batch."""

    def __init__(self, chunk_bytes: int = 256 << 20, world: int = 1, rank: int = 0):
        self.chunk = int(chunk_bytes)
        self.world, self.proc = world, rank

    def run(self, ranks, layout: DistLayout, gq: int, stream_ctx=None) -> None:
        import torch

        j = gq - layout.m
        half_of = {}
        for r in ranks.ranks:
            view = ranks.bytes_view(r)
            h = view.numel() // 2
            top = 1 - ((r >> j) & 1)  # the half that leaves this rank
            half_of[r] = view[top * h:(top + 1) * h]
        h = next(iter(half_of.values())).numel()
        ctx = stream_ctx() if stream_ctx else _null()
        with ctx:
            p2p = []
            for r in ranks.ranks:
                p = r ^ (1 << j)
                if p in half_of:
                    if r < p:
                        self._swap_local(half_of[r], half_of[p])
                    continue
                p2p.append((r, p))
            if p2p:
                self._swap_remote(half_of, p2p, layout, h)

    def _swap_local(self, a, b) -> None:
        import torch

        step = min(self.chunk, a.numel())
        tmp = torch.empty(step, dtype=a.dtype, device=a.device)
        for o in range(0, a.numel(), step):
            e = min(o + step, a.numel())
            t = tmp[: e - o]
            t.copy_(a[o:e])
            a[o:e].copy_(b[o:e])
            b[o:e].copy_(t)

    def _swap_remote(self, half_of, pairs, layout: DistLayout, h: int) -> None:
        import torch
        import torch.distributed as dist

        step = min(self.chunk, h)
        bufs = {r: torch.empty(step, dtype=half_of[r].dtype, device=half_of[r].device) for r, _ in pairs}
        for o in range(0, h, step):
            e = min(o + step, h)
            ops = []
            for r, p in pairs:
                peer = owner(p, layout, self.world)
                ops.append(dist.P2POp(dist.isend, half_of[r][o:e], peer, tag=p))
                ops.append(dist.P2POp(dist.irecv, bufs[r][: e - o], peer, tag=r))
            for w in dist.batch_isend_irecv(ops):
                w.wait()
            for r, _ in pairs:
                half_of[r][o:e].copy_(bufs[r][: e - o])


class _null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


# ---- running a plan -------------------------------------------------------------------------------
@dataclass
class DistState:
    plan: DistPlan
    ranks: object
    world: int = 1
    proc: int = 0
    stats: dict = field(default_factory=dict)


def execute(plan: DistPlan, ranks, exchange: Exchange, stream_ctx: Callable | None = None) -> DistState:
    """Runs ``plan`` from |0...0> on this process's ranks (``EngineRanks``,
    or any object with the same methods)."""
    layout = plan.layout
    n_ex = 0
    for step in plan.steps:
        if isinstance(step, LocalStep):
            for r in ranks.ranks:
                ranks.apply(r, rank_program(step.instructions, layout, r))
        else:
            exchange.run(ranks, layout, step.global_qubit, stream_ctx)
            n_ex += 1
    state = DistState(plan, ranks, exchange.world, exchange.proc, {"exchanges": n_ex, "steps": len(plan.steps)})
    if getattr(ranks, "renormalizes", lambda: False)():
        # the single-node TC32 stream ends with a rescale to norm 1; over
        # ranks the norm is the sum of the slices' norms
        total = norm_sqr(state)
        if total > 0.0:
            for r in ranks.ranks:
                ranks.scale(r, 1.0 / np.sqrt(total))
        ranks.be.set_tuning("renormalize", 1)  # the handle's own streams rescale again
    return state


def run_distributed(circuit: C.Circuit, g: int, backend, world: int = 1, rank: int = 0,
                    chunk_bytes: int = 256 << 20) -> DistState:
    """The circuit over 2^g ranks of this engine: this process runs its block
    of ranks (all of them when world = 1) on the backend's GPU; exchanges
    with ranks of other processes go over the default process group."""
    layout = DistLayout(circuit.num_qubits, g)
    if layout.ranks % world:
        raise DistError(f"{layout.ranks} ranks do not split over {world} processes")
    per = layout.ranks // world
    plan = plan_dist(circuit.instructions, layout)
    ranks = EngineRanks(backend, layout, range(rank * per, (rank + 1) * per))
    return execute(plan, ranks, Exchange(chunk_bytes, world, rank), ranks.stream_ctx)


def gather_statevector(state: DistState) -> np.ndarray:
    """The full state in logical qubit order (all ranks on this process;
    small n): physical index p holds logical index x with bit q of x at
    position final_map[q]."""
    layout = state.plan.layout
    phys = np.concatenate([state.ranks.statevector(r) for r in range(layout.ranks)])
    return unmap(phys, state.plan.final_map)


def unmap(phys: np.ndarray, final_map: Sequence[int]) -> np.ndarray:
    n = len(final_map)
    x = np.arange(1 << n, dtype=np.int64)
    p = np.zeros_like(x)
    for q, pq in enumerate(final_map):
        p |= ((x >> q) & 1) << pq
    return phys[p]


def norm_sqr(state: DistState) -> float:
    """sum |a|^2 over every rank: per-rank device reductions, summed over the
    processes (all-reduce) when there is more than one."""
    s = sum(state.ranks.norm_sqr(r) for r in state.ranks.ranks)
    if state.world > 1:
        import torch
        import torch.distributed as dist

        t = torch.tensor([s], dtype=torch.float64)
        if dist.get_backend() == "nccl":
            t = t.cuda()
        dist.all_reduce(t)
        s = float(t.item())
    return s
