"""Seeded random circuits shared by the parity tests (GPU engine and CPU pipeline)."""
import numpy as np

from aleph_b200 import circuit as C
from aleph_b200 import workloads


def random_circuit(n, depth, seed):
    """Every gate variant, with and without generic controls."""
    rng = np.random.default_rng(seed)
    c = C.Circuit(n)
    one = ["H", "X", "Y", "Z", "S", "Sdg", "T", "Tdg"]
    par1 = ["Rx", "Ry", "Rz", "Phase"]
    two = ["Cnot", "Cz", "Swap", "Iswap", "IswapDg"]
    par2 = ["CRx", "CRy", "CRz"]
    for _ in range(depth):
        kind = rng.integers(0, 10)
        qs = [int(x) for x in rng.permutation(n)[:5]]
        ctrl = [qs[4]] if rng.random() < 0.25 and n > 4 else []
        if kind == 0:
            c.add(C.Gate(str(rng.choice(one))), [qs[0]], ctrl)
        elif kind == 1:
            c.add(C.Gate(str(rng.choice(par1)), (float(rng.uniform(-7, 7)),)), [qs[0]], ctrl)
        elif kind == 2:
            c.add(C.U3(*rng.uniform(-4, 4, 3)), [qs[0]], ctrl)
        elif kind == 3:
            c.add(C.Gate(str(rng.choice(two))), qs[:2], ctrl)
        elif kind == 4:
            c.add(C.Gate(str(rng.choice(par2)), (float(rng.uniform(-7, 7)),)), qs[:2], ctrl)
        elif kind == 5:
            c.add(C.Gate(str(rng.choice(["Toffoli", "Ccz"]))), qs[:3], ctrl)
        elif kind == 6:
            c.add(C.Unitary1q(workloads.haar_su2(rng)), [qs[0]], ctrl)
        elif kind == 7:
            z = rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4))
            q, _ = np.linalg.qr(z)
            c.add(C.Unitary2q(q), qs[:2], ctrl)
        elif kind == 8:
            k = int(rng.integers(2, 6))
            z = rng.standard_normal((2**k, 2**k)) + 1j * rng.standard_normal((2**k, 2**k))
            q, _ = np.linalg.qr(z)
            c.add(C.UnitaryKq(q), qs[:k])
        else:
            ph = np.exp(1j * rng.uniform(0, 6.3, 4))
            if rng.random() < 0.5:
                c.add(C.Unitary1qDiag(ph[:2]), [qs[0]], ctrl)
            else:
                c.add(C.Unitary2qDiag(ph), qs[:2], ctrl)
    return c
