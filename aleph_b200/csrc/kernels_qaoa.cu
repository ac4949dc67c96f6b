// kernels_qaoa.cu — batched QAOA Max-Cut sweep: many parameter sets with
// ragged qubit counts in one persistent launch.
//
// Circuit of one set (build_qaoa, crates/aleph-ir/src/ansatz.rs:71-98): H on
// every qubit, then p layers of [CNOT(i,j) Rz(2 gamma)_j CNOT(i,j) per edge,
// Rx(2 beta) on every qubit]. On a basis state z the edge gadget is the phase
// exp(-i gamma (1 - 2 [z_i != z_j])), so a cost layer is the diagonal
// exp(-i gamma (m - 2 cut(z))) with m edges; a mixer layer is Rx(2 beta) on
// every qubit. The output is <C> = sum_z |psi_z|^2 cut(z), the expectation of
// H_C = sum_edges 1/2 (I - Z_i Z_j) (ansatz.rs:100-117), reduced in FP64.
//
// One CTA per SM pulls sets from a queue (largest first). A state of at most
// SMEM_N qubits lives in shared memory for the whole circuit. A larger one
// lives in the CTA's slice of a device buffer and is streamed in tiles of
// 2^13 amplitudes, two passes per layer: pass A over contiguous chunks
// (qubits 0..12: cost phase + mixer), pass B over tiles spanning the qubits
// 13..n-1 (mixer). The first pass generates |+>^n instead of reading it; the
// last pass only reads and accumulates <C>. A pass loads a tile into
// registers (32 amplitudes a thread, every load in flight at once), mixes the
// register and lane bits there, and at most one trip through shared memory
// mixes the warp bits.
//
// cut(z) per amplitude: within a pass-A chunk z = (t << 13) | lo and
// cut(z) = cutT[lo] + (edges among the high qubits cut by t) + X0[lo & 127] +
// X1[lo >> 7], where cutT counts the edges among qubits 0..12 (per set) and
// X0 / X1 the edges between a low and a high qubit (per chunk). The first
// cost layer also stores cut(z) as one byte per amplitude, which the final
// pass B reads. Multiple edges between the same pair count once each, as the
// repeated gadgets do.

#include "common.cuh"

namespace ab {

namespace qaoa {

constexpr int THREADS = 256;
constexpr int TILE_BITS = 13;
constexpr uint32_t TILE = 1u << TILE_BITS;
constexpr int MAX_EDGES = 128;
template <typename Real>
struct Cfg {
  static constexpr int SMEM_N = 13;  // states kept in shared memory (the tile size)
  static constexpr uint32_t SMEM_BYTES = (1u << SMEM_N) * sizeof(V2<Real>);
  // FP32 tiles (64 KiB) leave room for two CTAs per SM, which overlap one
  // CTA's tile loads with the other's arithmetic
  static constexpr int CTAS_PER_SM = sizeof(Real) == 4 ? 2 : 1;
};

struct Args {
  const aleph_b200_qaoa_set* sets;
  const uint32_t* edges;   // (u, v) pairs
  const double* angles;    // per set: gamma[0..p), beta[0..p)
  const uint32_t* order;   // set indices, largest first
  uint32_t* next;          // work counter (zero at launch)
  double* out;
  void* scratch;           // per-CTA state slices for the streamed sets
  uint8_t* cuts;           // per-CTA cut(z) slices
  uint64_t slice_amps;
  uint32_t n_sets, p;
};

// Rx(2 beta) on tile-local bit k of every pair in S[0..len): (a, b) -> (c a - i s b, c b - i s a).
template <typename Real>
__device__ __forceinline__ void mixer_bit(V2<Real>* S, uint32_t len, uint32_t k, Real c, Real s) {
  for (uint32_t i = threadIdx.x; i < len / 2; i += THREADS) {
    const uint32_t j0 = (uint32_t)insert_zero(i, k), j1 = j0 | (1u << k);
    const V2<Real> a = S[j0], b = S[j1];
    S[j0] = mk<Real>(c * a.x + s * b.y, c * a.y - s * b.x);
    S[j1] = mk<Real>(c * b.x + s * a.y, c * b.y - s * a.x);
  }
}

// Rx(2 beta) on tile-local bits k0 < k1 of every quartet: one shared-memory
// sweep for two qubits (the four amplitudes of a quartet in registers).
template <typename Real>
__device__ __forceinline__ void mixer_bits2(V2<Real>* S, uint32_t len, uint32_t k0, uint32_t k1, Real c, Real s) {
  auto rx = [&](V2<Real>& a, V2<Real>& b) {
    const V2<Real> x = a, y = b;
    a = mk<Real>(c * x.x + s * y.y, c * x.y - s * y.x);
    b = mk<Real>(c * y.x + s * x.y, c * y.y - s * x.x);
  };
  for (uint32_t i = threadIdx.x; i < len / 4; i += THREADS) {
    const uint32_t e00 = (uint32_t)insert_zero(insert_zero(i, k0), k1);
    const uint32_t e01 = e00 | (1u << k0), e10 = e00 | (1u << k1), e11 = e01 | (1u << k1);
    V2<Real> a00 = S[e00], a01 = S[e01], a10 = S[e10], a11 = S[e11];
    rx(a00, a01);
    rx(a10, a11);
    rx(a00, a10);
    rx(a01, a11);
    S[e00] = a00;
    S[e01] = a01;
    S[e10] = a10;
    S[e11] = a11;
  }
}

// Rx on the tile-local bits first, first+1, ..., first+count-1: two per sweep.
template <typename Real>
__device__ __forceinline__ void mixer_range(V2<Real>* S, uint32_t len, uint32_t first, uint32_t count, Real c, Real s) {
  uint32_t k = 0;
  for (; k + 1 < count; k += 2) {
    __syncthreads();
    mixer_bits2<Real>(S, len, first + k, first + k + 1, c, s);
  }
  if (k < count) {
    __syncthreads();
    mixer_bit<Real>(S, len, first + k, c, s);
  }
  __syncthreads();
}

// Streamed tiles are swept in registers. Register layout: tile index
// i = tid | r << 8 (lane = tile bits 0..4, warp = bits 5..7, register r =
// bits 8..12), so one thread issues all REGS of its loads before it uses one.
constexpr int REGS = TILE / THREADS;
static_assert(THREADS == 256 && REGS == 32, "the sweep layouts assume 8 warps and 32 registers");

template <typename Real>
__device__ __forceinline__ void rx_pair(V2<Real>& a, V2<Real>& b, Real c, Real s) {
  const V2<Real> x = a, y = b;
  a = mk<Real>(c * x.x + s * y.y, c * x.y - s * y.x);
  b = mk<Real>(c * y.x + s * x.y, c * y.y - s * x.x);
}

// Rx(2 beta) on register bit k of v for every k set in mask.
template <typename Real, int NR>
__device__ __forceinline__ void rx_regs(V2<Real> (&v)[NR], uint32_t mask, Real c, Real s) {
#pragma unroll
  for (int k = 0; (1 << k) < NR; ++k) {
    if (!((mask >> k) & 1u)) continue;
#pragma unroll
    for (int r = 0; r < NR; ++r)
      if (!(r & (1 << k))) rx_pair<Real>(v[r], v[r | (1 << k)], c, s);
  }
}

// Rx(2 beta) on lane bit k for every k set in mask (uniform across the warp):
// the partner amplitude comes from lane ^ (1 << k), and both halves of a pair
// take the same form x' = c x - i s y.
template <typename Real, int NR>
__device__ __forceinline__ void rx_lanes(V2<Real> (&v)[NR], uint32_t mask, Real c, Real s) {
  // FP32: the lane bit is a runtime shuffle mask, so a rolled loop keeps one
  // copy of the body (unrolled, the FP32 sweeps stall on instruction fetch;
  // rolled they ran 4% faster). FP64 keeps it unrolled (2% faster so).
#pragma unroll(sizeof(Real) == 4 ? 1 : 5)
  for (int k = 0; k < 5; ++k) {
    if (!((mask >> k) & 1u)) continue;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const Real yx = __shfl_xor_sync(0xffffffffu, v[r].x, 1 << k);
      const Real yy = __shfl_xor_sync(0xffffffffu, v[r].y, 1 << k);
      v[r] = mk<Real>(c * v[r].x + s * yy, c * v[r].y - s * yx);
    }
  }
}

// One read of the tile in shared memory in the layout lane = tile bits 0..4,
// register = bits 5..7, warp and loop = bits 8..12: Rx on the register bits
// set in mask3, then emit(i, amplitude) for each of this thread's 32 indices.
template <typename Real, typename Emit>
__device__ __forceinline__ void shared_sweep(const V2<Real>* S, uint32_t mask3, Real c, Real s, Emit&& emit) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint32_t hi = (w | (uint32_t)j << 3) << 8;
    V2<Real> u[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) u[r] = S[hi | (uint32_t)r << 5 | lane];
    rx_regs<Real, 8>(u, mask3, c, s);
#pragma unroll
    for (int r = 0; r < 8; ++r) emit(hi | (uint32_t)r << 5 | lane, u[r]);
  }
}

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < THREADS / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

template <typename Real>
__global__ void __launch_bounds__(THREADS, Cfg<Real>::CTAS_PER_SM) sweep_kernel(Args a) {
  extern __shared__ __align__(16) uint8_t qsm[];
  V2<Real>* S = (V2<Real>*)qsm;
  __shared__ uint8_t eu[MAX_EDGES], ev[MAX_EDGES];
  __shared__ uint8_t cutT[1 << TILE_BITS];
  __shared__ uint8_t X0[128], X1[64];
  __shared__ V2<Real> ph[MAX_EDGES + 1];  // cost-layer phase by cut value
  __shared__ double red[THREADS / 32];
  __shared__ uint32_t s_idx, s_ch;
  const uint32_t tid = threadIdx.x;
  V2<Real>* X = (V2<Real>*)a.scratch + (uint64_t)blockIdx.x * a.slice_amps;
  uint8_t* CG = a.cuts + (uint64_t)blockIdx.x * a.slice_amps;

  for (;;) {
    if (tid == 0) s_idx = atomicAdd(a.next, 1u);
    __syncthreads();
    const uint32_t idx = s_idx;
    __syncthreads();
    if (idx >= a.n_sets) break;
    const uint32_t ci = a.order[idx];
    const aleph_b200_qaoa_set cs = a.sets[ci];
    const uint32_t n = cs.num_qubits, m = cs.num_edges;
    for (uint32_t e = tid; e < m; e += THREADS) {
      eu[e] = (uint8_t)a.edges[2 * (cs.edge_offset + e)];
      ev[e] = (uint8_t)a.edges[2 * (cs.edge_offset + e) + 1];
    }
    __syncthreads();
    const bool in_smem = n <= (uint32_t)Cfg<Real>::SMEM_N;
    const uint32_t lb = in_smem ? n : (uint32_t)TILE_BITS;  // cutT covers qubits 0..lb-1
    for (uint32_t z = tid; z < (1u << lb); z += THREADS) {
      uint32_t c = 0;
      for (uint32_t e = 0; e < m; ++e)
        if (eu[e] < lb && ev[e] < lb) c += ((z >> eu[e]) ^ (z >> ev[e])) & 1u;
      cutT[z] = (uint8_t)c;
    }
    const double* gam = a.angles + (size_t)ci * 2 * a.p;
    const double* bet = gam + a.p;
    const uint64_t len = 1ull << n;
    const Real amp0 = (Real)rsqrt((double)len);  // |+>^n
    auto set_phases = [&](double gamma) {  // ph[k] = exp(-i gamma (m - 2k))
      __syncthreads();
      for (uint32_t k = tid; k <= m; k += THREADS) {
        double sn, cn;
        sincos(-gamma * ((double)m - 2.0 * (double)k), &sn, &cn);
        ph[k] = mk<Real>((Real)cn, (Real)sn);
      }
      __syncthreads();
    };
    double acc = 0.0;

    if (in_smem) {
      // ---- whole state in shared memory ----
      const uint32_t L = (uint32_t)len;
      for (uint32_t i = tid; i < L; i += THREADS) S[i] = mk<Real>(amp0, (Real)0);
      for (uint32_t l = 0; l < a.p; ++l) {
        set_phases(gam[l]);
        for (uint32_t i = tid; i < L; i += THREADS) S[i] = cmul<Real>(ph[cutT[i]], S[i]);
        double sb, cb;
        sincos(bet[l], &sb, &cb);
        mixer_range<Real>(S, L, 0, n, (Real)cb, (Real)sb);
      }
      for (uint32_t i = tid; i < L; i += THREADS) {
        const double x = (double)S[i].x, y = (double)S[i].y;
        acc += (x * x + y * y) * (double)cutT[i];
      }
    } else {
      // ---- streamed through this CTA's state slice ----
      const uint32_t c = 2 * TILE_BITS - n;                 // pass B: low run bits (n <= 26)
      const uint32_t maskB = (TILE - 1) & ~((1u << c) - 1);  // pass B mixes tile bits c..12
      const uint64_t ntiles = len >> TILE_BITS;
      V2<Real> v[REGS];  // the register sweep's amplitudes (see load_chunk / load_tile)
      for (uint32_t l = 0; l < a.p; ++l) {
        set_phases(gam[l]);
        double sb, cb;
        sincos(bet[l], &sb, &cb);
        const Real rc = (Real)cb, rs = (Real)sb;
        // pass A: contiguous chunks, cost phase + mixer on qubits 0..12.
        // Chunk constants: cut edges among the high qubits, and the low/high
        // cross-edge tables.
        auto chunk_tables = [&](uint32_t t) {
          if (tid == 0) {
            uint32_t ch = 0;
            for (uint32_t e = 0; e < m; ++e)
              if (eu[e] >= TILE_BITS && ev[e] >= TILE_BITS)
                ch += (uint32_t)(((t >> (eu[e] - TILE_BITS)) ^ (t >> (ev[e] - TILE_BITS))) & 1u);
            s_ch = ch;
          }
          if (tid < 192) {
            const uint32_t base = tid < 128 ? 0u : 7u, v = tid < 128 ? tid : tid - 128;
            uint32_t x = 0;
            for (uint32_t e = 0; e < m; ++e) {
              const uint32_t u0 = eu[e], v0 = ev[e];
              const bool ul = u0 < TILE_BITS, vl = v0 < TILE_BITS;
              if (ul == vl) continue;  // not a low/high cross edge
              const uint32_t lo_q = ul ? u0 : v0, hi_q = ul ? v0 : u0;
              if (lo_q < base || lo_q >= base + (base ? 6u : 7u)) continue;
              const uint32_t zb = (v >> (lo_q - base)) & 1u, hb = (uint32_t)(t >> (hi_q - TILE_BITS)) & 1u;
              x += zb ^ hb;
            }
            if (tid < 128) X0[v] = (uint8_t)x;
            else X1[v] = (uint8_t)x;
          }
        };
        // this thread's 32 amplitudes i = tid | r << 8 of chunk t, every load in flight at once
        // (slice offsets fit in 32 bits: n <= 26)
        auto load_chunk = [&](uint32_t t) {
          if (l == 0) {
#pragma unroll
            for (int r = 0; r < REGS; ++r) v[r] = mk<Real>(amp0, (Real)0);
          } else {
#pragma unroll
            for (int r = 0; r < REGS; ++r) v[r] = X[(t << TILE_BITS) | tid | (uint32_t)r << 8];
          }
        };
        // Software pipeline: chunk t+1's loads and tables are issued once chunk
        // t sits in shared memory, and are in flight during its shared sweep.
        chunk_tables(0);
        load_chunk(0);
        for (uint32_t t = 0; t < (uint32_t)ntiles; ++t) {
          __syncthreads();  // chunk t's tables are visible; chunk t-1's shared sweep is done
          const uint32_t ch = s_ch;
          const uint32_t g0 = t << TILE_BITS;
          const uint32_t x0 = X0[tid & 127];
#pragma unroll
          for (int r = 0; r < REGS; ++r) {
            const uint32_t i = tid | (uint32_t)r << 8;
            const uint32_t cut = cutT[i] + ch + x0 + X1[i >> 7];
            if (l == 0) CG[g0 + i] = (uint8_t)cut;
            v[r] = cmul<Real>(ph[cut], v[r]);
          }
          rx_regs<Real, REGS>(v, 0x1fu, rc, rs);   // tile bits 8..12
          rx_lanes<Real, REGS>(v, 0x1fu, rc, rs);  // tile bits 0..4
#pragma unroll
          for (int r = 0; r < REGS; ++r) S[tid | (uint32_t)r << 8] = v[r];
          __syncthreads();
          if (t + 1 < (uint32_t)ntiles) {
            chunk_tables(t + 1);
            load_chunk(t + 1);
          }
          // shared-memory sweep: tile bits 5..7, straight back to the chunk
          shared_sweep<Real>(S, 0x7u, rc, rs, [&](uint32_t i, const V2<Real>& u) { X[g0 + i] = u; });
        }
        __syncthreads();  // pass A's stores are visible to every thread of the CTA
        // pass B: tiles over {qubits 0..c-1} + {qubits 13..n-1}; tile index -> qubits c..12
        const bool last = l + 1 == a.p;
        const uint32_t lowm = (1u << c) - 1;
        auto gidx = [&](uint32_t t, uint32_t i) -> uint32_t {
          return (i & lowm) | t << c | (i >> c) << TILE_BITS;
        };
        auto load_tile = [&](uint32_t t) {
#pragma unroll
          for (int r = 0; r < REGS; ++r) v[r] = X[gidx(t, tid | (uint32_t)r << 8)];
        };
        load_tile(0);
        for (uint32_t t = 0; t < (uint32_t)ntiles; ++t) {
          rx_regs<Real, REGS>(v, maskB >> 8, rc, rs);
          rx_lanes<Real, REGS>(v, maskB & 0x1fu, rc, rs);
          __syncthreads();  // the previous tile's shared-memory sweep is done
#pragma unroll
          for (int r = 0; r < REGS; ++r) S[tid | (uint32_t)r << 8] = v[r];
          __syncthreads();
          if (t + 1 < (uint32_t)ntiles) load_tile(t + 1);
          shared_sweep<Real>(S, (maskB >> 5) & 0x7u, rc, rs, [&](uint32_t i, const V2<Real>& u) {
            if (last) {
              const double x = (double)u.x, y = (double)u.y;
              acc += (x * x + y * y) * (double)CG[gidx(t, i)];
            } else {
              X[gidx(t, i)] = u;
            }
          });
        }
      }
    }
    const double tot = block_sum(acc, red);
    if (tid == 0) a.out[ci] = tot;
    __syncthreads();
  }
}

}  // namespace qaoa

uint32_t qaoa_smem_max_n(int precision) {
  return precision == ALEPH_B200_F64 ? (uint32_t)qaoa::Cfg<double>::SMEM_N : (uint32_t)qaoa::Cfg<float>::SMEM_N;
}

int qaoa_ctas_per_sm(int precision) {
  return precision == ALEPH_B200_F64 ? qaoa::Cfg<double>::CTAS_PER_SM : qaoa::Cfg<float>::CTAS_PER_SM;
}

cudaError_t launch_qaoa_sweep(int precision, const aleph_b200_qaoa_set* sets, const uint32_t* edges,
                              const double* angles, const uint32_t* order, uint32_t* next, double* out,
                              void* scratch, uint8_t* cuts, uint64_t slice_amps, uint32_t n_sets, uint32_t p,
                              int grid, cudaStream_t s) {
  qaoa::Args a{sets, edges, angles, order, next, out, scratch, cuts, slice_amps, n_sets, p};
  static uint64_t attr_devices[2] = {0, 0};  // per precision: devices with the shared-memory opt-in
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const int k = precision == ALEPH_B200_F64 ? 1 : 0;
  if (dev >= 64 || !((attr_devices[k] >> dev) & 1)) {
    e = k ? cudaFuncSetAttribute(qaoa::sweep_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 qaoa::Cfg<double>::SMEM_BYTES)
          : cudaFuncSetAttribute(qaoa::sweep_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 qaoa::Cfg<float>::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    if (dev < 64) attr_devices[k] |= 1ull << dev;
  }
  if (k)
    qaoa::sweep_kernel<double><<<grid, qaoa::THREADS, qaoa::Cfg<double>::SMEM_BYTES, s>>>(a);
  else
    qaoa::sweep_kernel<float><<<grid, qaoa::THREADS, qaoa::Cfg<float>::SMEM_BYTES, s>>>(a);
  return cudaGetLastError();
}

}  // namespace ab
