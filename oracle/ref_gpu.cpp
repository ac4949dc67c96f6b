// ref_gpu.cpp — REFERENCE ARM, test and bench infrastructure, not product code.
//
// Runs the reference's own CUDA state-vector kernels on this machine's GPU, so
// that the engine can be timed against the reference's GPU design on the same
// device. The kernels are the reference's sources, compiled unchanged by
// oracle/Makefile (target `ref`) into oracle/_ref/*.cubin:
//   crates/aleph-cuda/src/sv/kernels.cu      (FP64: apply_1q, apply_1q_multi,
//                                             apply_cnot, apply_phase_poly,
//                                             apply_kq, apply_kq_tiled)
//   crates/aleph-cuda/src/sv/diag.cu         (FP64: apply_diag_1q, apply_diag)
//   crates/aleph-cuda/src/sv/kernels_f32.cu  (FP32: the same set, `_f32`)
// This file is the host side the reference writes in Rust, restated: the
// per-gate parameter structs (byte layouts of crates/aleph-cuda/src/sv/kernel.rs
// and diag.rs), the launch shapes (256-thread blocks, one thread per pair /
// group / amplitude) and the dispatch of CudaSvBackend::run_layered
// (crates/aleph-cuda/src/sv/backend.rs:515-575), apply_gate (:678-757) and
// the FP32 twin (crates/aleph-cuda/src/sv/fp32.rs:425-495). The instruction
// stream comes already planned by the reference's CUDA pass list
// (orc_gpu_pipeline_plan in sv_pipeline.cpp).
//
// The CUDA driver is opened with dlopen on first use, so this library still
// loads on a machine without a GPU driver.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda.h>

#include "../include/aleph_b200.h"

extern "C" int orc_gate_matrix(const aleph_b200_instr* g, const double* pool, uint64_t pool_len, double* out,
                               int* dim_out);

namespace {

// ---- the driver entry points this harness uses -------------------------------------
struct Driver {
  CUresult (*Init)(unsigned);
  CUresult (*DeviceGet)(CUdevice*, int);
  CUresult (*PrimaryCtxRetain)(CUcontext*, CUdevice);
  CUresult (*CtxSetCurrent)(CUcontext);
  CUresult (*ModuleLoad)(CUmodule*, const char*);
  CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*);
  CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                           void**, void**);
  CUresult (*MemAlloc)(CUdeviceptr*, size_t);
  CUresult (*MemFree)(CUdeviceptr);
  CUresult (*MemcpyHtoDAsync)(CUdeviceptr, const void*, size_t, CUstream);
  CUresult (*MemcpyDtoH)(void*, CUdeviceptr, size_t);
  CUresult (*MemsetD8Async)(CUdeviceptr, unsigned char, size_t, CUstream);
  CUresult (*MemAllocAsync)(CUdeviceptr*, size_t, CUstream);
  CUresult (*MemFreeAsync)(CUdeviceptr, CUstream);
  CUresult (*StreamCreate)(CUstream*, unsigned);
  CUresult (*StreamSynchronize)(CUstream);
  CUresult (*StreamDestroy)(CUstream);
  CUresult (*EventCreate)(CUevent*, unsigned);
  CUresult (*EventRecord)(CUevent, CUstream);
  CUresult (*EventSynchronize)(CUevent);
  CUresult (*EventElapsedTime)(float*, CUevent, CUevent);
  CUresult (*EventDestroy)(CUevent);
  CUresult (*GetErrorString)(CUresult, const char**);
};

Driver D;
bool g_driver = false;
std::string g_err;

template <typename F>
bool sym(void* h, const char* name, F* f) {
  *f = reinterpret_cast<F>(dlsym(h, name));
  if (!*f) g_err = std::string("missing driver symbol ") + name;
  return *f != nullptr;
}

bool open_driver() {
  if (g_driver) return true;
  void* h = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
  if (!h) {
    g_err = "libcuda.so.1 not found";
    return false;
  }
  bool ok = sym(h, "cuInit", &D.Init) && sym(h, "cuDeviceGet", &D.DeviceGet) &&
            sym(h, "cuDevicePrimaryCtxRetain", &D.PrimaryCtxRetain) && sym(h, "cuCtxSetCurrent", &D.CtxSetCurrent) &&
            sym(h, "cuModuleLoad", &D.ModuleLoad) && sym(h, "cuModuleGetFunction", &D.ModuleGetFunction) &&
            sym(h, "cuLaunchKernel", &D.LaunchKernel) && sym(h, "cuMemAlloc_v2", &D.MemAlloc) &&
            sym(h, "cuMemFree_v2", &D.MemFree) && sym(h, "cuMemcpyHtoDAsync_v2", &D.MemcpyHtoDAsync) &&
            sym(h, "cuMemcpyDtoH_v2", &D.MemcpyDtoH) && sym(h, "cuMemsetD8Async", &D.MemsetD8Async) &&
            sym(h, "cuMemAllocAsync", &D.MemAllocAsync) && sym(h, "cuMemFreeAsync", &D.MemFreeAsync) &&
            sym(h, "cuStreamCreate", &D.StreamCreate) && sym(h, "cuStreamSynchronize", &D.StreamSynchronize) &&
            sym(h, "cuStreamDestroy_v2", &D.StreamDestroy) && sym(h, "cuEventCreate", &D.EventCreate) &&
            sym(h, "cuEventRecord", &D.EventRecord) && sym(h, "cuEventSynchronize", &D.EventSynchronize) &&
            sym(h, "cuEventElapsedTime", &D.EventElapsedTime) && sym(h, "cuEventDestroy_v2", &D.EventDestroy) &&
            sym(h, "cuGetErrorString", &D.GetErrorString);
  g_driver = ok;
  return ok;
}

bool check(CUresult r, const char* what) {
  if (r == CUDA_SUCCESS) return true;
  const char* s = nullptr;
  if (D.GetErrorString) D.GetErrorString(r, &s);
  g_err = std::string(what) + ": " + (s ? s : "CUDA error");
  return false;
}

// ---- parameter structs: byte layouts of the reference's kernel uniforms -----------
// (crates/aleph-cuda/src/sv/kernel.rs:36-130, diag.rs:29-64)
struct Gate1q {
  double m[8];  // m00 m01 m10 m11, interleaved (re, im)
  uint32_t target, t_bit, ctrl_mask, pad;
};
struct GateKq {
  uint32_t k, qbit[5], sorted[5], ctrl_mask;
};
struct Multi1q {
  double mats[40];  // gate j: mats[8j .. 8j+8)
  uint32_t m, sorted[5], pad[2];
};
struct Cnot {
  uint32_t ctrl, targ, lo, hi;
};
struct Diag1q {
  double d0[2], d1[2];
  uint32_t t_bit, ctrl_mask;
};
struct DiagK {
  uint32_t k, qbit[5], ctrl_mask;
};
static_assert(sizeof(Gate1q) == 80 && sizeof(GateKq) == 48 && sizeof(Multi1q) == 352 && sizeof(Cnot) == 16 &&
                  sizeof(Diag1q) == 40 && sizeof(DiagK) == 28,
              "kernel uniform layouts");

constexpr unsigned kBlock = 256;       // BLOCK (backend.rs:29, diag.rs:23)
constexpr size_t kLayerBatch = 3;      // DEFAULT_LAYER_BATCH (kernel.rs:30)
constexpr uint32_t kTiledMinK = 2;     // tiled_min_k default (backend.rs:127)
constexpr double kAmplitudeTol = 1e-10;  // aleph_core::AMPLITUDE_TOL (diagonal_of, common.rs:56-79)

enum Fn { F1Q, FMULTI, FCNOT, FPOLY, FKQ, FKQT, FDIAG1, FDIAG, NFN };
const char* kNames[NFN] = {"apply_1q", "apply_1q_multi", "apply_cnot", "apply_phase_poly",
                           "apply_kq", "apply_kq_tiled", "apply_diag_1q", "apply_diag"};

struct Modules {
  bool loaded = false;
  CUfunction f[2][NFN];  // [f32][fn]
};
Modules g_mod;
CUcontext g_ctx = nullptr;

bool load_modules(const char* dir) {
  if (g_mod.loaded) return true;
  if (!open_driver()) return false;
  CUdevice dev;
  if (!check(D.Init(0), "cuInit") || !check(D.DeviceGet(&dev, 0), "cuDeviceGet") ||
      !check(D.PrimaryCtxRetain(&g_ctx, dev), "cuDevicePrimaryCtxRetain") ||
      !check(D.CtxSetCurrent(g_ctx), "cuCtxSetCurrent"))
    return false;
  CUmodule m64, mdiag, m32;
  const std::string d(dir);
  if (!check(D.ModuleLoad(&m64, (d + "/sv_kernels.cubin").c_str()), "load sv_kernels.cubin") ||
      !check(D.ModuleLoad(&mdiag, (d + "/sv_diag.cubin").c_str()), "load sv_diag.cubin") ||
      !check(D.ModuleLoad(&m32, (d + "/sv_kernels_f32.cubin").c_str()), "load sv_kernels_f32.cubin"))
    return false;
  for (int i = 0; i < NFN; ++i) {
    CUmodule m = (i == FDIAG1 || i == FDIAG) ? mdiag : m64;
    if (!check(D.ModuleGetFunction(&g_mod.f[0][i], m, kNames[i]), kNames[i])) return false;
    const std::string n32 = std::string(kNames[i]) + "_f32";
    if (!check(D.ModuleGetFunction(&g_mod.f[1][i], m32, n32.c_str()), n32.c_str())) return false;
  }
  g_mod.loaded = true;
  return true;
}

// One run of a planned stream on one state: the reference's run_layered.
struct Runner {
  uint32_t n;
  int f32;
  CUstream s;
  CUdeviceptr amps;
  CUdeviceptr scratch;  // mat_scratch: the largest dense matrix, 32 x 32 complex
  const aleph_b200_pools* pools;
  uint64_t launches = 0;

  bool launch(Fn fn, uint64_t threads, void** args, unsigned shared = 0) {
    const uint64_t blocks = std::max<uint64_t>(1, (threads + kBlock - 1) / kBlock);
    ++launches;
    return check(D.LaunchKernel(g_mod.f[f32][fn], (unsigned)blocks, 1, 1, kBlock, 1, 1, shared, s, args, nullptr),
                 kNames[fn]);
  }
  static uint32_t ctrl_mask(const aleph_b200_instr& r) {
    uint32_t m = 0;
    for (uint32_t i = 0; i < r.num_controls; ++i) m |= 1u << r.controls[i];
    return m;
  }
  // gate_kq_params (backend.rs:624-640): matrix bit b <-> qubits[k-1-b]
  static GateKq kq_params(const uint32_t* q, uint32_t k, uint32_t cmask) {
    GateKq p{};
    p.k = k;
    for (uint32_t b = 0; b < k; ++b) p.qbit[b] = 1u << q[k - 1 - b];
    for (uint32_t b = 0; b < k; ++b) p.sorted[b] = q[b];
    std::sort(p.sorted, p.sorted + k);
    p.ctrl_mask = cmask;
    return p;
  }
  bool upload_scratch(const double* m, size_t doubles) {
    return check(D.MemcpyHtoDAsync(scratch, m, doubles * sizeof(double), s), "matrix upload");
  }
  // launch_kq / launch_kq_tiled (backend.rs:247-327)
  bool kq(GateKq p, const double* mat) {
    const uint32_t dim = 1u << p.k;
    if (!upload_scratch(mat, 2ull * dim * dim)) return false;
    if (p.k >= kTiledMinK) {
      uint64_t n_amps = 1ull << n;
      void* args[] = {&amps, &scratch, &p, &n_amps};
      return launch(FKQT, n_amps, args, dim * dim * (f32 ? 8 : 16));  // the matrix as cplx / cplxf
    }
    uint64_t groups = 1ull << (n - p.k);
    void* args[] = {&amps, &scratch, &p, &groups};
    return launch(FKQ, groups, args);
  }
  // apply_1q_layer (backend.rs:468-501): chunks of DEFAULT_LAYER_BATCH, each
  // sorted by qubit, one apply_1q_multi sweep per chunk
  bool layer(const std::vector<std::pair<uint32_t, std::vector<double>>>& gates) {
    for (size_t c0 = 0; c0 < gates.size(); c0 += kLayerBatch) {
      const size_t m = std::min(kLayerBatch, gates.size() - c0);
      std::vector<size_t> idx(m);
      for (size_t i = 0; i < m; ++i) idx[i] = c0 + i;
      std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return gates[a].first < gates[b].first; });
      Multi1q p{};
      p.m = (uint32_t)m;
      for (size_t j = 0; j < m; ++j) {
        p.sorted[j] = gates[idx[j]].first;
        std::memcpy(p.mats + 8 * j, gates[idx[j]].second.data(), 8 * sizeof(double));
      }
      uint64_t groups = 1ull << (n - m);
      void* args[] = {&amps, &p, &groups};
      if (!launch(FMULTI, groups, args)) return false;
    }
    return true;
  }
  // launch_phase_poly (backend.rs:362-419): CSR upload, one sweep
  bool phase_poly(const aleph_b200_instr& r) {
    if (r.data_len == 0) return true;
    std::vector<double> angles;
    std::vector<uint64_t> conds;
    std::vector<uint32_t> offsets{0};
    for (uint64_t t = 0; t < r.data_len; ++t) {
      const aleph_b200_phase_term& pt = pools->terms[r.data_offset + t];
      angles.push_back(pt.angle);
      for (uint32_t c = 0; c < pt.cond_count; ++c) conds.push_back(pools->cond_pool[pt.cond_offset + c]);
      offsets.push_back((uint32_t)conds.size());
    }
    if (conds.empty()) conds.push_back(0);
    CUdeviceptr da, dc, dofs;
    if (!check(D.MemAllocAsync(&da, angles.size() * 8, s), "alloc") ||
        !check(D.MemAllocAsync(&dc, conds.size() * 8, s), "alloc") ||
        !check(D.MemAllocAsync(&dofs, offsets.size() * 4, s), "alloc"))
      return false;
    bool ok = check(D.MemcpyHtoDAsync(da, angles.data(), angles.size() * 8, s), "upload") &&
              check(D.MemcpyHtoDAsync(dc, conds.data(), conds.size() * 8, s), "upload") &&
              check(D.MemcpyHtoDAsync(dofs, offsets.data(), offsets.size() * 4, s), "upload");
    if (ok) {
      uint32_t nt = (uint32_t)r.data_len;
      uint64_t n_amps = 1ull << n;
      void* args[] = {&amps, &da, &dc, &dofs, &nt, &n_amps};
      ok = launch(FPOLY, n_amps, args);
    }
    D.MemFreeAsync(da, s);
    D.MemFreeAsync(dc, s);
    D.MemFreeAsync(dofs, s);
    return ok;
  }
  // apply_gate (backend.rs:678-757; fp32.rs:425-495)
  bool gate(const aleph_b200_instr& r) {
    const uint32_t cm = ctrl_mask(r);
    if (r.kind == ALEPH_GATE_CNOT && r.num_controls == 0 && r.num_qubits == 2) {
      Cnot p{r.qubits[0], r.qubits[1], std::min(r.qubits[0], r.qubits[1]), std::max(r.qubits[0], r.qubits[1])};
      uint64_t groups = 1ull << (n - 2);
      void* args[] = {&amps, &p, &groups};
      return launch(FCNOT, groups, args);
    }
    if (r.kind == ALEPH_GATE_UNITARYKQ) {
      std::vector<double> m(pools->matrix_pool + 2 * r.data_offset, pools->matrix_pool + 2 * (r.data_offset + r.data_len));
      return kq(kq_params(r.qubits, r.aux, cm), m.data());
    }
    double mat[128];
    int dim = 0;
    if (orc_gate_matrix(&r, pools->matrix_pool, pools->matrix_pool_len, mat, &dim) != 0 || dim < 2) {
      g_err = "gate matrix";
      return false;
    }
    bool diag = true;  // diagonal_of: every off-diagonal entry within AMPLITUDE_TOL
    for (int i = 0; i < dim && diag; ++i)
      for (int j = 0; j < dim; ++j)
        if (i != j && std::hypot(mat[2 * (i * dim + j)], mat[2 * (i * dim + j) + 1]) > kAmplitudeTol) diag = false;
    const uint32_t k = (uint32_t)__builtin_ctz((unsigned)dim);
    if (diag) {
      uint64_t n_amps = 1ull << n;
      if (k == 1) {
        Diag1q p{{mat[0], mat[1]}, {mat[6], mat[7]}, 1u << r.qubits[0], cm};
        void* args[] = {&amps, &p, &n_amps};
        return launch(FDIAG1, n_amps, args);
      }
      std::vector<double> d;
      for (int i = 0; i < dim; ++i) {
        d.push_back(mat[2 * (i * dim + i)]);
        d.push_back(mat[2 * (i * dim + i) + 1]);
      }
      if (!upload_scratch(d.data(), d.size())) return false;
      DiagK p{};
      p.k = k;
      for (uint32_t b = 0; b < k; ++b) p.qbit[b] = 1u << r.qubits[k - 1 - b];
      p.ctrl_mask = cm;
      void* args[] = {&amps, &scratch, &p, &n_amps};
      return launch(FDIAG, n_amps, args);
    }
    if (k == 1) {
      Gate1q p{};
      std::memcpy(p.m, mat, sizeof(p.m));
      p.target = r.qubits[0];
      p.t_bit = 1u << r.qubits[0];
      p.ctrl_mask = cm;
      uint64_t pairs = 1ull << (n - 1);
      void* args[] = {&amps, &p, &pairs};
      return launch(F1Q, pairs, args);
    }
    return kq(kq_params(r.qubits, k, cm), mat);
  }
  // run_layered (backend.rs:515-575): plain one-qubit gates collect into a
  // pending layer (flushed on a repeated qubit and before anything else)
  bool run(const aleph_b200_instr* in, uint64_t count) {
    std::vector<std::pair<uint32_t, std::vector<double>>> pending;
    uint64_t mask = 0;
    auto flush = [&]() {
      bool ok = pending.empty() || layer(pending);
      pending.clear();
      mask = 0;
      return ok;
    };
    for (uint64_t i = 0; i < count; ++i) {
      const aleph_b200_instr& r = in[i];
      if (r.kind < 28) {
        double mat[128];
        int dim = 0;
        const bool batchable = r.num_qubits == 1 && r.num_controls == 0 && r.kind != ALEPH_GATE_UNITARYKQ &&
                               orc_gate_matrix(&r, pools->matrix_pool, pools->matrix_pool_len, mat, &dim) == 0 &&
                               dim == 2;
        if (batchable) {
          const uint64_t bit = 1ull << r.qubits[0];
          if ((mask & bit) && !flush()) return false;
          mask |= bit;
          pending.emplace_back(r.qubits[0], std::vector<double>(mat, mat + 8));
          continue;
        }
        if (!flush() || !gate(r)) return false;
      } else if (r.kind == ALEPH_INSTR_BARRIER) {
        if (!flush()) return false;
      } else if (r.kind == ALEPH_INSTR_DIAGONAL_PHASE) {
        if (!flush() || !phase_poly(r)) return false;
      } else {
        g_err = "instruction not supported by the reference arm";
        return false;
      }
    }
    return flush();
  }
};

}  // namespace

extern "C" {

/* Last error of the reference arm (driver message or dispatch error). */
const char* orc_refgpu_error() { return g_err.c_str(); }

/* Loads the compiled reference kernels from `dir` (sv_kernels.cubin,
 * sv_diag.cubin, sv_kernels_f32.cubin) on device 0. 0 on success. */
int orc_refgpu_load(const char* dir) { return load_modules(dir) ? 0 : -1; }

/* Runs the planned stream `repeats` times on a fresh |0...0> state of n qubits
 * (complex128, or complex64 when f32), each run timed with driver events on
 * one stream: ms[r] = run r. launches_out = kernel launches of one run. When
 * amps_out is given, the final state is copied to it as complex128. */
int orc_refgpu_run(uint32_t n, int f32, const aleph_b200_instr* instrs, uint64_t count, const aleph_b200_pools* pools,
                   int repeats, double* ms, uint64_t* launches_out, double* amps_out) {
  if (!g_mod.loaded) {
    g_err = "reference kernels not loaded";
    return -1;
  }
  if (n < 2 || n > (f32 ? 31u : 30u)) {  // MAX_CUDA_QUBITS 30 / MAX_CUDA_QUBITS_F32 31
    g_err = "qubit count outside the reference's CUDA range";
    return -1;
  }
  if (!check(D.CtxSetCurrent(g_ctx), "cuCtxSetCurrent")) return -1;
  const size_t amp_bytes = f32 ? 8 : 16;
  const size_t bytes = amp_bytes << n;
  Runner R{n, f32, nullptr, 0, 0, pools};
  CUevent e0 = nullptr, e1 = nullptr;
  int rc = -1;
  if (!check(D.StreamCreate(&R.s, CU_STREAM_NON_BLOCKING), "stream") ||
      !check(D.MemAlloc(&R.amps, bytes), "state alloc") || !check(D.MemAlloc(&R.scratch, 32 * 32 * 16), "alloc") ||
      !check(D.EventCreate(&e0, CU_EVENT_DEFAULT), "event") || !check(D.EventCreate(&e1, CU_EVENT_DEFAULT), "event"))
    goto done;
  for (int rep = 0; rep < repeats; ++rep) {
    // |0...0> (CudaSvState::allocate): zero fill plus amplitude 0 = 1
    const double one64[2] = {1.0, 0.0};
    const float one32[2] = {1.0f, 0.0f};
    if (!check(D.MemsetD8Async(R.amps, 0, bytes, R.s), "memset") ||
        !check(D.MemcpyHtoDAsync(R.amps, f32 ? (const void*)one32 : (const void*)one64, amp_bytes, R.s), "init") ||
        !check(D.StreamSynchronize(R.s), "sync"))
      goto done;
    R.launches = 0;
    if (!check(D.EventRecord(e0, R.s), "record") || !R.run(instrs, count) || !check(D.EventRecord(e1, R.s), "record") ||
        !check(D.EventSynchronize(e1), "run"))
      goto done;
    float t = 0;
    if (!check(D.EventElapsedTime(&t, e0, e1), "elapsed")) goto done;
    if (ms) ms[rep] = t;
  }
  if (launches_out) *launches_out = R.launches;
  if (amps_out) {
    if (f32) {
      std::vector<float> h((size_t)2 << n);
      if (!check(D.MemcpyDtoH(h.data(), R.amps, bytes), "read state")) goto done;
      for (size_t i = 0; i < h.size(); ++i) amps_out[i] = h[i];
    } else if (!check(D.MemcpyDtoH(amps_out, R.amps, bytes), "read state")) {
      goto done;
    }
  }
  rc = 0;
done:
  if (R.s) D.StreamSynchronize(R.s);
  if (e0) D.EventDestroy(e0);
  if (e1) D.EventDestroy(e1);
  if (R.scratch) D.MemFree(R.scratch);
  if (R.amps) D.MemFree(R.amps);
  if (R.s) D.StreamDestroy(R.s);
  return rc;
}

}  // extern "C"
