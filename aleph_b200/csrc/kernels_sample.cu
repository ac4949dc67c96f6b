// kernels_sample.cu — on-device shot sampling with the reference's exact
// seed-to-outcome mappings, given the same variates.
//
// ALIAS (the reference's shots >= 2 path, crates/aleph-sv/src/measure.rs:109-124):
//   probabilities p_i = re*re + im*im rounded exactly like the CPU (no FMA),
//   Vose's table built by AliasTable::build (crates/aleph-sv/src/sampling.rs:104-167)
//   with the same LIFO stack discipline and the same floating-point operation
//   order, so the table is bit-identical; the table build's sequential chain
//   runs on one thread (it is inherently sequential), the O(N) partition and
//   all draws run in parallel. Draw: index = (word >> 32) & (N-1),
//   u = (u32)word * 2^-32, u < prob[i] ? i : alias[i] (sampling.rs:179-197).
// CUMULATIVE (the reference's shots <= 1 path, sampling.rs:59-91): the
//   inverse CDF of the sequential left-to-right prefix sum with strict
//   `target < cumulative`, zero bins skipped, last positive bin as fallback.
//   Shots are resolved in parallel on a two-level prefix (tree block sums +
//   a sequential scan inside the block); a shot whose target lies within the
//   rounding bound of a bin boundary is re-resolved against the exact
//   sequential running sum (for n <= 28), so the outcome equals the
//   sequential CPU result.

#include <cmath>

#include "common.cuh"

namespace ab {

constexpr uint32_t CUM_BLOCK = 2048;  // amplitudes per level-1 CDF block
constexpr uint32_t EXACT_MAX_N = kExactCumulativeMaxN;  // exact re-resolution of ambiguous shots up to this n

template <typename Real>
__device__ __forceinline__ double prob_exact(const V2<Real>* amps, uint64_t i) {
  const V2<Real> a = ld_amp<Real>(amps + i);
  const double x = (double)a.x, y = (double)a.y;
  return __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
}

// ------------------------------------------------------------------ ALIAS ----
struct AliasScratch {
  double* prob;       // N: scaled probabilities, then the table thresholds
  uint32_t* alias;    // N
  uint32_t* small;    // N: indices with scaled < 1, ascending
  uint32_t* large;    // N: indices with scaled >= 1, ascending
  uint32_t* bcount;   // 2 * nb: per-block small / large counts, then exclusive offsets
  uint32_t* totals;   // 2: small / large counts
  double* normsum;    // 2 * nb partial [sum p, non-finite]
};

constexpr uint32_t PART_B = 1024;  // elements per partition block

template <typename Real>
__global__ void alias_scale_kernel(const V2<Real>* __restrict__ amps, uint64_t len, AliasScratch s) {
  // one block per PART_B elements: scaled values + per-block small/large counts + norm partials
  __shared__ uint32_t cs[32], cl[32];
  __shared__ double ns[32], nb[32];
  const double nf = (double)len;
  const uint64_t i = (uint64_t)blockIdx.x * PART_B + threadIdx.x;
  uint32_t small = 0, large = 0;
  double psum = 0.0, bad = 0.0;
  if (i < len) {
    const double p = prob_exact<Real>(amps, i);
    if (!isfinite(p)) bad = 1.0;
    else psum = p;
    const double sc = __dmul_rn(nf, p);
    s.prob[i] = sc;
    if (sc < 1.0) small = 1;
    else large = 1;
  }
  const unsigned bs = __ballot_sync(0xffffffffu, small), bl = __ballot_sync(0xffffffffu, large);
  for (int o = 16; o; o >>= 1) {
    psum += __shfl_down_sync(0xffffffffu, psum, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    cs[w] = __popc(bs);
    cl[w] = __popc(bl);
    ns[w] = psum;
    nb[w] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t a = 0, b = 0;
    double x = 0.0, y = 0.0;
    for (int k = 0; k < (int)(PART_B / 32); ++k) {
      a += cs[k];
      b += cl[k];
      x += ns[k];
      y += nb[k];
    }
    s.bcount[2 * blockIdx.x] = a;
    s.bcount[2 * blockIdx.x + 1] = b;
    s.normsum[2 * blockIdx.x] = x;
    s.normsum[2 * blockIdx.x + 1] = y;
  }
}

// Exclusive scan of the per-block counts (one thread; nb <= 2^18 blocks).
__global__ void alias_offsets_kernel(AliasScratch s, uint32_t nblocks, double* norm_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t a = 0, b = 0;
  double x = 0.0, y = 0.0;
  for (uint32_t k = 0; k < nblocks; ++k) {
    const uint32_t ca = s.bcount[2 * k], cb = s.bcount[2 * k + 1];
    s.bcount[2 * k] = a;
    s.bcount[2 * k + 1] = b;
    a += ca;
    b += cb;
    x += s.normsum[2 * k];
    y += s.normsum[2 * k + 1];
  }
  s.totals[0] = a;
  s.totals[1] = b;
  norm_out[0] = x;
  norm_out[1] = y;
}

__global__ void alias_partition_kernel(uint64_t len, AliasScratch s) {
  __shared__ uint32_t ws[32], wl[32];
  const uint64_t i = (uint64_t)blockIdx.x * PART_B + threadIdx.x;
  bool is_small = false, valid = i < len;
  if (valid) is_small = s.prob[i] < 1.0;
  const unsigned bs = __ballot_sync(0xffffffffu, valid && is_small);
  const unsigned bl = __ballot_sync(0xffffffffu, valid && !is_small);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    ws[w] = __popc(bs);
    wl[w] = __popc(bl);
  }
  __syncthreads();
  uint32_t os = s.bcount[2 * blockIdx.x], ol = s.bcount[2 * blockIdx.x + 1];
  for (int k = 0; k < w; ++k) {
    os += ws[k];
    ol += wl[k];
  }
  const unsigned below = (1u << lane) - 1u;
  if (valid) {
    if (is_small) s.small[os + __popc(bs & below)] = (uint32_t)i;
    else s.large[ol + __popc(bl & below)] = (uint32_t)i;
  }
}

// The Vose loop of AliasTable::build, one warp.
//
// With LIFO stacks, the element pushed in one step is popped in the next: a
// large whose residual stays >= 1 is the next large, one that drops below 1
// is the next small. So that element lives in lane 0's registers, and the
// stacks themselves are only ever popped: their entries below the top, and
// the scaled values of those entries, are read-only until popped. The warp
// therefore streams them into shared-memory buffers ahead of the chain
// (descending stack order), and lane 0 runs the dependent chain out of
// shared memory with the reference's operation order,
//   alias[s] = l, threshold[s] = value(s), value(l) = (value(l) + value(s)) - 1.
// status[0] is set on failure (never expected: the rounds are bounded).
// Lane 0's step is the add / subtract / compare and selects, without
// data-dependent branches: the next entry of each buffer sits in registers one
// step ahead (the buffers carry one spare slot so that this read never leaves
// them), and each step's outputs (alias[s] = l, threshold[s]) go to a
// shared-memory record ring that the whole warp scatters to global memory
// when it fills or a buffer runs dry.
constexpr int CHAIN_CH = 1024;
constexpr int REC_CAP = 1024;
__global__ void __launch_bounds__(32) alias_chain_kernel(uint64_t len, AliasScratch s, int32_t* status) {
  __shared__ uint32_t sbi[CHAIN_CH + 1], lbi[CHAIN_CH + 1];
  __shared__ double sbv[CHAIN_CH + 1], lbv[CHAIN_CH + 1];
  __shared__ uint32_t rec_s[REC_CAP], rec_l[REC_CAP];
  __shared__ double rec_v[REC_CAP];
  const int lane = threadIdx.x;
  if (len == 1) {
    if (lane == 0) {
      s.prob[0] = 1.0;
      s.alias[0] = 0;
    }
    return;
  }
  int64_t ts = (int64_t)s.totals[0];  // small entries not yet buffered: small[0..ts)
  int64_t tl = (int64_t)s.totals[1];  // large entries not yet buffered: large[0..tl)
  int ns = 0, ps = 0, nl = 0, pl = 0;  // buffer fill / consumed counts (uniform over the warp)
  bool hs = false, hl = false;         // lane 0: current small / large held in registers
  uint32_t si = 0, li = 0;
  double sv = 0.0, lv = 0.0;
  uint64_t guard = 0;
  int fail = 0;
  while (true) {
    if (ps == ns && ts > 0) {  // refill the small buffer from the stack top
      const int m = ts < CHAIN_CH ? (int)ts : CHAIN_CH;
      for (int k = lane; k < m; k += 32) {
        const uint32_t id = s.small[ts - 1 - k];
        sbi[k] = id;
        sbv[k] = s.prob[id];
      }
      ts -= m;
      ns = m;
      ps = 0;
    }
    if (pl == nl && tl > 0) {
      const int m = tl < CHAIN_CH ? (int)tl : CHAIN_CH;
      for (int k = lane; k < m; k += 32) {
        const uint32_t id = s.large[tl - 1 - k];
        lbi[k] = id;
        lbv[k] = s.prob[id];
      }
      tl -= m;
      nl = m;
      pl = 0;
    }
    __syncwarp();
    int done = 0, nrec = 0;
    if (lane == 0) {
      if (++guard > 4 * (len / 256) + 64) fail = 1;  // rounds: refills plus ring flushes
      if (!hs && ps < ns) {
        si = sbi[ps];
        sv = sbv[ps];
        ++ps;
        hs = true;
      }
      if (!hl && pl < nl) {
        li = lbi[pl];
        lv = lbv[pl];
        ++pl;
        hl = true;
      }
      if (hs && hl && !fail) {
        // next entries of each buffer (meaningful while ps < ns / pl < nl)
        uint32_t nsi = sbi[ps], nli = lbi[pl];
        double nsv = sbv[ps], nlv = lbv[pl];
        while (true) {
          rec_s[nrec] = si;
          rec_l[nrec] = li;
          rec_v[nrec] = sv;  // threshold = value of the small
          ++nrec;
          const double r = __dsub_rn(__dadd_rn(lv, sv), 1.0);
          const bool t = r < 1.0;  // the large becomes the next small
          if (t ? pl >= nl : ps >= ns) {  // its successor is not buffered yet
            if (t) {
              si = li;
              sv = r;
              hl = false;
            } else {
              lv = r;
              hs = false;
            }
            break;
          }
          const uint32_t si2 = t ? li : nsi, li2 = t ? nli : li;
          const double sv2 = t ? r : nsv, lv2 = t ? nlv : r;
          si = si2;
          li = li2;
          sv = sv2;
          lv = lv2;
          ps += t ? 0 : 1;
          pl += t ? 1 : 0;
          nsi = sbi[ps];
          nsv = sbv[ps];
          nli = lbi[pl];
          nlv = lbv[pl];
          if (nrec == REC_CAP) break;  // the warp flushes the ring first
        }
      }
      done = fail || (!hs && ps == ns && ts == 0) || (!hl && pl == nl && tl == 0);
    }
    ps = __shfl_sync(0xffffffffu, ps, 0);
    pl = __shfl_sync(0xffffffffu, pl, 0);
    done = __shfl_sync(0xffffffffu, done, 0);
    nrec = __shfl_sync(0xffffffffu, nrec, 0);
    __syncwarp();
    for (int k = lane; k < nrec; k += 32) {  // scatter the step records
      s.alias[rec_s[k]] = rec_l[k];
      s.prob[rec_s[k]] = rec_v[k];
    }
    __syncwarp();
    if (done) break;
  }
  if (lane == 0) {
    if (fail) {
      status[0] = ALEPH_B200_DEVICE_FAILURE;
      return;
    }
    // Leftovers, drained below as self-aliases with threshold 1: the stack
    // entries never popped (still in memory below the buffered ones) plus the
    // element held in registers, pushed back on its stack.
    int64_t rs = ts + (ns - ps), rl = tl + (nl - pl);
    if (hs) s.small[rs++] = si;
    if (hl) s.large[rl++] = li;
    s.totals[0] = (uint32_t)rs;
    s.totals[1] = (uint32_t)rl;
  }
}

__global__ void alias_drain_kernel(AliasScratch s) {
  const uint32_t ts = s.totals[0], tl = s.totals[1];
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < ts + tl; k += gridDim.x * blockDim.x) {
    const uint32_t i = k < ts ? s.small[k] : s.large[k - ts];
    s.prob[i] = 1.0;
    s.alias[i] = i;
  }
}

__global__ void alias_draw_kernel(AliasScratch s, uint64_t mask, const uint64_t* __restrict__ words, uint32_t shots,
                                  uint64_t* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < shots; k += gridDim.x * blockDim.x) {
    const uint64_t bits = words[k];
    const uint64_t i = (bits >> 32) & mask;
    const double u = (double)(uint32_t)bits * (1.0 / 4294967296.0);
    out[k] = u < s.prob[i] ? i : (uint64_t)s.alias[i];
  }
}

// Norm check of validate_state (sampling.rs:36-57): sets status on failure.
__global__ void check_norm_kernel(const double* norm2, double tol, int32_t* status) {
  if (threadIdx.x != 0) return;
  const double total = norm2[0];
  if (norm2[1] > 0.0 || !isfinite(total) || fabs(total - 1.0) > tol)
    status[0] = ALEPH_B200_INVALID_STATE;
}

// ------------------------------------------------------------- CUMULATIVE ----
struct CumScratch {
  double* bsum;      // nb + 1: block sums, then exclusive block prefix (bsum[nb] = total)
  double* norm;      // 2: [total, non-finite count]
  uint32_t* namb;    // ambiguous shot count
  uint32_t* amb;     // shots: ambiguous shot ids
  double* ck;        // exact mode: sequential sum at the end of every SEQ_CH chunk
  double* seq;       // exact mode: [sequential total, last positive index (bits)]
};

template <typename Real>
__global__ void cum_blocks_kernel(const V2<Real>* __restrict__ amps, uint64_t len, CumScratch c) {
  __shared__ double red[2][8];
  const uint64_t b0 = (uint64_t)blockIdx.x * CUM_BLOCK;
  double x = 0.0, bad = 0.0;
  for (uint32_t j = threadIdx.x; j < CUM_BLOCK && b0 + j < len; j += blockDim.x) {
    const double p = prob_exact<Real>(amps, b0 + j);
    if (isfinite(p)) x += p;
    else bad += 1.0;
  }
  for (int o = 16; o; o >>= 1) {
    x += __shfl_down_sync(0xffffffffu, x, o);
    bad += __shfl_down_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = x;
    red[1][threadIdx.x >> 5] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      s += red[0][w];
      b += red[1][w];
    }
    c.bsum[blockIdx.x] = s;
    if (b > 0.0) atomicAdd(&c.norm[1], b);
  }
}

// Exclusive prefix of the block sums, one CTA of PREFIX_T threads: thread t
// sums a contiguous range, the range totals are scanned in shared memory, and
// each thread writes its range's prefixes. The draws treat this prefix as an
// approximation (guard band E below), so its rounding order is free.
constexpr uint32_t PREFIX_T = 1024;
__global__ void __launch_bounds__(PREFIX_T) cum_prefix_kernel(CumScratch c, uint32_t nb) {
  __shared__ double part[PREFIX_T];
  const uint32_t t = threadIdx.x;
  const uint32_t per = (nb + PREFIX_T - 1) / PREFIX_T;
  const uint32_t b0 = min(nb, t * per), b1 = min(nb, b0 + per);
  double s = 0.0;
  for (uint32_t b = b0; b < b1; ++b) s += c.bsum[b];
  part[t] = s;
  __syncthreads();
  for (uint32_t off = 1; off < PREFIX_T; off <<= 1) {  // inclusive Hillis-Steele scan
    const double v = t >= off ? part[t - off] : 0.0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  double run = t ? part[t - 1] : 0.0;
  for (uint32_t b = b0; b < b1; ++b) {
    const double x = c.bsum[b];
    c.bsum[b] = run;
    run += x;
  }
  if (t == PREFIX_T - 1) {
    c.bsum[nb] = part[PREFIX_T - 1];
    c.norm[0] = part[PREFIX_T - 1];
  }
}

template <typename Real>
__global__ void cum_draw_kernel(const V2<Real>* __restrict__ amps, uint64_t len, uint32_t nb, CumScratch c,
                                const double* __restrict__ uniforms, uint32_t shots, uint64_t* __restrict__ out,
                                int32_t* status) {
  const double total = c.bsum[nb];
  // Bound on |sequential - two-level| for prefixes and for u * total.
  const double E = 8.0 * ((double)len + 64.0) * 1.1102230246251565e-16 * total;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < shots; k += gridDim.x * blockDim.x) {
    const double target = uniforms[k] * total;
    // last block whose exclusive prefix <= target
    uint32_t lo = 0, hi = nb;  // invariant: prefix[lo] <= target (prefix[0] = 0)
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (c.bsum[mid] <= target) lo = mid;
      else hi = mid;
    }
    double cum = c.bsum[lo];
    double margin = fabs(target - cum);
    int64_t found = -1, last_pos = -1;
    for (uint64_t i = (uint64_t)lo * CUM_BLOCK; i < len; ++i) {
      const double p = prob_exact<Real>(amps, i);
      if (p > 0.0) {
        last_pos = (int64_t)i;
        cum += p;
        margin = fmin(margin, fabs(cum - target));
        if (target < cum) {
          found = (int64_t)i;
          break;
        }
      }
    }
    if (found < 0) {
      // ran off the end: the last positive bin at or after the start block,
      // or, if none, any earlier positive bin (resolved exactly below)
      found = last_pos;
      margin = 0.0;
    }
    out[k] = (uint64_t)(found < 0 ? 0 : found);
    if (margin <= E) {
      const uint32_t slot = atomicAdd(c.namb, 1u);
      c.amb[slot] = k;
    }
  }
}

// Exact resolution of the ambiguous shots, in two kernels.
//
// cum_seq_kernel: the reference's sequential left-to-right sum
// (validate_norm's total and cumulative_index's running sum are the same
// sequence S_i = fl(S_{i-1} + p_i)), done once by one thread while the rest
// of the CTA stages the next chunk of probabilities in shared memory. It
// records S at the end of every SEQ_CH-element chunk (exact checkpoints),
// the total and the last positive index.
// cum_exact_kernel: per ambiguous shot, the first chunk whose checkpoint
// exceeds the target, rescanned sequentially from the previous checkpoint,
// so every outcome equals the sequential CPU scan's.
constexpr uint32_t SEQ_CH = 2048;
constexpr uint32_t SEQ_T = 512;

template <typename Real>
__global__ void __launch_bounds__(SEQ_T) cum_seq_kernel(const V2<Real>* __restrict__ amps, uint64_t len, CumScratch c) {
  __shared__ double buf[2][SEQ_CH];
  if (*c.namb == 0) return;  // uniform over the CTA: no ambiguous shot, nothing to resolve
  const uint64_t nch = (len + SEQ_CH - 1) / SEQ_CH;
  auto stage = [&](uint64_t ch, int slot) {
    const uint64_t b0 = ch * SEQ_CH;
    for (uint32_t j = threadIdx.x; j < SEQ_CH; j += SEQ_T)
      buf[slot][j] = b0 + j < len ? prob_exact<Real>(amps, b0 + j) : 0.0;
  };
  stage(0, 0);
  __syncthreads();
  double S = 0.0;
  int64_t last_pos = -1;
  for (uint64_t ch = 0; ch < nch; ++ch) {
    if (threadIdx.x == 0) {
      const double* b = buf[ch & 1];
      const uint64_t left = len - ch * SEQ_CH;
      const uint32_t m = left < SEQ_CH ? (uint32_t)left : SEQ_CH;
#pragma unroll 16
      for (uint32_t j = 0; j < m; ++j) {
        const double p = b[j];
        S += p;
        if (p > 0.0) last_pos = (int64_t)(ch * SEQ_CH + j);
      }
      c.ck[ch] = S;
    } else if (ch + 1 < nch) {
      // threads 1.. stage the next chunk (thread 0's share falls to the others)
      const uint64_t b0 = (ch + 1) * SEQ_CH;
      for (uint32_t j = threadIdx.x - 1; j < SEQ_CH; j += SEQ_T - 1)
        buf[(ch + 1) & 1][j] = b0 + j < len ? prob_exact<Real>(amps, b0 + j) : 0.0;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    c.seq[0] = S;
    c.seq[1] = __longlong_as_double(last_pos);
  }
}

template <typename Real>
__global__ void cum_exact_kernel(const V2<Real>* __restrict__ amps, uint64_t len, CumScratch c,
                                 const double* __restrict__ uniforms, uint64_t* __restrict__ out, int32_t* status) {
  const uint32_t na = *c.namb;
  const uint64_t nch = (len + SEQ_CH - 1) / SEQ_CH;
  const double total = c.seq[0];
  const int64_t last_pos = __double_as_longlong(c.seq[1]);
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < na; a += gridDim.x * blockDim.x) {
    const uint32_t k = c.amb[a];
    const double target = uniforms[k] * total;
    // first chunk whose inclusive checkpoint exceeds the target
    uint64_t lo = 0, hi = nch;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (target < c.ck[mid]) hi = mid;
      else lo = mid + 1;
    }
    if (lo == nch) {  // target >= total: the last positive bin
      if (last_pos < 0) status[0] = ALEPH_B200_INVALID_STATE;
      else out[k] = (uint64_t)last_pos;
      continue;
    }
    double S = lo ? c.ck[lo - 1] : 0.0;
    const uint64_t e = (lo + 1) * SEQ_CH < len ? (lo + 1) * SEQ_CH : len;
    for (uint64_t i = lo * SEQ_CH; i < e; ++i) {
      const double p = prob_exact<Real>(amps, i);
      if (p > 0.0) {
        S += p;
        if (target < S) {
          out[k] = i;
          break;
        }
      }
    }
  }
}

size_t sample_scratch_bytes(uint32_t n, int mode, uint32_t shots) {
  const uint64_t len = 1ull << n;
  if (mode == ALEPH_B200_SAMPLE_ALIAS) {
    const uint64_t nb = (len + PART_B - 1) / PART_B;
    return len * (8 + 4 + 4 + 4) + nb * (8 + 16) + 256;
  }
  const uint64_t nb = (len + CUM_BLOCK - 1) / CUM_BLOCK;
  const uint64_t nch = n <= EXACT_MAX_N ? (len + SEQ_CH - 1) / SEQ_CH : 0;  // exact-mode checkpoints
  return (nb + 1) * 8 + 64 + 256 + (size_t)shots * 4 + 16 + nch * 8 + 32;
}

static inline char* align_up(char* p, size_t a) {
  return (char*)(((uintptr_t)p + a - 1) & ~(uintptr_t)(a - 1));
}

cudaError_t launch_sample(const void* amps, int precision, uint32_t n, uint32_t shots, int mode, const void* variates,
                          uint64_t* out, void* scratch, size_t scratch_bytes, int32_t* status, int sm_count,
                          cudaStream_t st) {
  const uint64_t len = 1ull << n;
  const bool f64 = precision == ALEPH_B200_F64;
  char* p = (char*)scratch;
  if (mode == ALEPH_B200_SAMPLE_ALIAS) {
    const uint32_t nb = (uint32_t)((len + PART_B - 1) / PART_B);
    AliasScratch s;
    s.prob = (double*)p; p += len * 8;
    s.normsum = (double*)p; p += (size_t)nb * 16;
    s.alias = (uint32_t*)p; p += len * 4;
    s.small = (uint32_t*)p; p += len * 4;
    s.large = (uint32_t*)p; p += len * 4;
    s.bcount = (uint32_t*)p; p += (size_t)nb * 8;
    p = align_up(p, 16);
    s.totals = (uint32_t*)p; p += 16;
    double* norm2 = (double*)p; p += 16;
    if ((size_t)(p - (char*)scratch) > scratch_bytes) return cudaErrorInvalidValue;
    if (f64) alias_scale_kernel<double><<<nb, PART_B, 0, st>>>((const double2*)amps, len, s);
    else alias_scale_kernel<float><<<nb, PART_B, 0, st>>>((const float2*)amps, len, s);
    alias_offsets_kernel<<<1, 32, 0, st>>>(s, nb, norm2);
    check_norm_kernel<<<1, 32, 0, st>>>(norm2, norm_tolerance(len, precision), status);
    alias_partition_kernel<<<nb, PART_B, 0, st>>>(len, s);
    alias_chain_kernel<<<1, 32, 0, st>>>(len, s, status);
    alias_drain_kernel<<<(unsigned)sm_count * 4, 256, 0, st>>>(s);
    if (shots)
      alias_draw_kernel<<<(shots + 255) / 256, 256, 0, st>>>(s, len - 1, (const uint64_t*)variates, shots, out);
    return cudaGetLastError();
  }
  const uint32_t nb = (uint32_t)((len + CUM_BLOCK - 1) / CUM_BLOCK);
  CumScratch c;
  c.bsum = (double*)p; p += ((size_t)nb + 1) * 8;
  p = align_up(p, 16);
  c.norm = (double*)p; p += 16;
  c.namb = (uint32_t*)p; p += 16;
  c.amb = (uint32_t*)align_up(p, 16);
  p = (char*)(c.amb + shots);
  const uint64_t nch = n <= EXACT_MAX_N ? (len + SEQ_CH - 1) / SEQ_CH : 0;
  c.seq = (double*)align_up(p, 16); p = (char*)(c.seq + 2);
  c.ck = (double*)p; p += nch * 8;
  if ((size_t)(p - (char*)scratch) > scratch_bytes) return cudaErrorInvalidValue;
  cudaMemsetAsync(c.norm, 0, 32, st);
  if (f64) cum_blocks_kernel<double><<<nb, 256, 0, st>>>((const double2*)amps, len, c);
  else cum_blocks_kernel<float><<<nb, 256, 0, st>>>((const float2*)amps, len, c);
  cum_prefix_kernel<<<1, PREFIX_T, 0, st>>>(c, nb);
  check_norm_kernel<<<1, 32, 0, st>>>(c.norm, norm_tolerance(len, precision), status);
  if (shots) {
    if (f64)
      cum_draw_kernel<double><<<(shots + 127) / 128, 128, 0, st>>>((const double2*)amps, len, nb, c,
                                                                   (const double*)variates, shots, out, status);
    else
      cum_draw_kernel<float><<<(shots + 127) / 128, 128, 0, st>>>((const float2*)amps, len, nb, c,
                                                                  (const double*)variates, shots, out, status);
    // status[2]: the shots inside the guard band (re-resolved below when n <= EXACT_MAX_N)
    cudaMemcpyAsync(status + 2, c.namb, 4, cudaMemcpyDeviceToDevice, st);
    if (n <= EXACT_MAX_N) {
      const unsigned eb = (shots + 127) / 128;
      if (f64) {
        cum_seq_kernel<double><<<1, SEQ_T, 0, st>>>((const double2*)amps, len, c);
        cum_exact_kernel<double><<<eb, 128, 0, st>>>((const double2*)amps, len, c, (const double*)variates, out, status);
      } else {
        cum_seq_kernel<float><<<1, SEQ_T, 0, st>>>((const float2*)amps, len, c);
        cum_exact_kernel<float><<<eb, 128, 0, st>>>((const float2*)amps, len, c, (const double*)variates, out, status);
      }
    }
  }
  return cudaGetLastError();
}

// ---- fixed scratch of aleph_b200_sample_cumulative_noalloc ----------------------
// Reserved when this module is loaded on a device, so the entry point that
// uses it never allocates. One copy per device; calls that overlap on one
// device share it.
static __device__ __align__(256) unsigned char g_fixed_sample_scratch[kFixedSampleScratchBytes];

cudaError_t fixed_sample_scratch_address(void** out) {
  return cudaGetSymbolAddress(out, g_fixed_sample_scratch);
}

}  // namespace ab
