// Internal declarations shared by the libdisorder translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "common.cuh"
#include "fft.cuh"

// ---------------------------------------------------------------- context
struct disorder_ctx_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  char err[2048] = {0};
  long long launches = 0;
  int sm_count = 148;
  size_t smem_optin = 0;
  // cached workspaces: operator scratch, solver vectors, small reductions
  void* ws = nullptr;
  size_t ws_bytes = 0;
  void* ws2 = nullptr;
  size_t ws2_bytes = 0;
  void* small = nullptr;
  size_t small_bytes = 0;
  cudaEvent_t ev[16] = {};
  int* d_err = nullptr;  // device error word of bounded in-kernel waits (0: none)
  // pinned host words the solvers' reductions land in (one set per context:
  // contexts driven from different host threads must not share them)
  void* h_scalars = nullptr;
  // the static scratch array of disorder_sinc_rigid_transform_static on this
  // device, resolved at context creation (null if that failed)
  void* static_scratch = nullptr;
  size_t static_scratch_bytes = 0;
  int fault = 0;  // one-shot injected fault (disorder_ctx_inject_fault)
  int precision = DISORDER_PRECISION_FP32;  // tensor-core contractions (disorder_ctx_set_precision)
  int tune_tma = 1;  // strided line passes on TMA tiles (1) or cp.async pipelines (0) (disorder_ctx_set_tuning)
  int tune_coil = 0;  // coil stage: three passes (0) or sample sums (1) (disorder_ctx_set_tuning)
};

// Workspace bump allocator on top of the context's cached buffer.
struct Workspace {
  char* base = nullptr;
  size_t cap = 0;
  size_t off = 0;
  template <class T>
  T* take(size_t n) {
    size_t bytes = ((n * sizeof(T)) + 255) & ~size_t(255);
    if (off + bytes > cap) return nullptr;
    T* p = reinterpret_cast<T*>(base + off);
    off += bytes;
    return p;
  }
};
int dis_workspace(disorder_ctx_s* ctx, size_t bytes, Workspace* ws);   // operator scratch
int dis_workspace2(disorder_ctx_s* ctx, size_t bytes, Workspace* ws);  // solver vectors
int dis_small(disorder_ctx_s* ctx, Workspace* ws);                     // 16 MB reduction scratch

// ---------------------------------------------------------------- plan
struct disorder_plan_s {
  disorder_ctx_s* ctx = nullptr;
  int N[3] = {0, 0, 0};
  long long V = 0;
  FFTPlan fft[3];
  std::vector<float> rG[3], kG[3];
  float cent[3] = {0, 0, 0};
  float* d_kG[3] = {nullptr, nullptr, nullptr};
  float* d_rG[3] = {nullptr, nullptr, nullptr};
  int n_seg = 0, n_mot = 0;
  long long n_samples = 0;
  std::vector<long long> seg_off;
  // samples, device
  int* d_ky = nullptr;
  int* d_kz = nullptr;
  // per-segment CSR over ky rows: samples of segment s with row ky are
  // d_perm[d_rowptr[s*(N1+1)+ky] .. d_rowptr[s*(N1+1)+ky+1])
  int* d_rowptr = nullptr;
  int* d_perm = nullptr;
  int* d_kyq = nullptr;     // ky, kz of the sample at each CSR position
  int* d_kzq = nullptr;
  int* d_seg_of = nullptr;  // segment of each sample
  long long* d_seg_off = nullptr;
  float2* d_tw[3] = {nullptr, nullptr, nullptr};  // exp(-2 pi i m / N[axis]), m < N[axis]
  // kG[axis][k] = k_alpha * (k < N/2 ? k : k - N) to within 4 ulp (even N)
  double k_alpha[3] = {0, 0, 0};
  bool k_linear[3] = {false, false, false};
};

// true unless DISORDER_GENERIC_FFT=1 forces the generic shared-memory kernels
bool dis_use_fast();
// true unless DISORDER_NO_PIPE=1 keeps every pass on the one-tile-per-CTA kernels
bool dis_use_pipe();

// ---------------------------------------------------------------- line pass
enum { P_ZERO = 0, P_A = 1, P_B = 2, P_ONE = 3, P_DK = 4 };

struct TabRef {
  const float2* p = nullptr;  // [slot][row][k]
  long long sstride = 0;      // elements per slot
  int b = -1;                 // axis whose coordinate selects the row (-1: 1-D table)
};

struct LinePassArgs {
  int N[3];
  int axis;
  int L;
  int pitch;
  int n_slots;
  int accumulate;   // out0 = beta*out0 + sum over slots (one grid.y)
  float beta;
  const float2* in0;
  long long in0_s;
  const float2* in1;
  long long in1_s;
  float2* out0;
  long long out0_s;
  float2* out1;
  long long out1_s;
  TabRef A, B, T;
  int c00, c01, c10, c11;
  // Per-row phase seeds of the whole coefficient (c00 times T) for the
  // pipelined kernel, [slot][row][sd_w] (tables.cu, seed_table_kernel);
  // Sd.p == nullptr: use A and T.
  TabRef Sd;
  int sd_w;
  const float* kG;  // device kGrid along the axis (P_DK)
  const float2* tw;  // device twiddle table of the axis
  FFTPlan plan;
};

int dis_line_pass(disorder_ctx_s* ctx, LinePassArgs a);

// flipping (Methods/flipping.m) of selected slots, in place, along one axis
int dis_flip_pass(disorder_ctx_s* ctx, const disorder_plan_s* plan, float2* vols, long long vstride,
                  const int* d_slots, int n_slots, int axis, float cent);

// ---------------------------------------------------------------- tables
// Per-slot transform parameters computed on the host in double precision.
struct SlotParams {
  double t[3];     // (-1)^di * T(1:3)   (phase of e1 is i*t*k)
  double tau[3];   // (-1)^(di-1) * tan(theta/2)   (phase of e2 is i*tau*rk1)
  double sig[3];   // (-1)^di * sin(theta)          (phase of e3 is i*sig*rk2)
  double g2[3];    // (1+tan^2(theta/2))/2     (etg2 = i*g2*rk1*e2)
  double g3[3];    // cos(theta)               (etg3 = -i*g3*rk2*e3)
  int flip[3];
};

struct Tables {
  // e2[m], e3[m], (etg2[m], etg3[m]) : [slot][row][k] with 1/N of the pass axis folded in
  float2* e2[3] = {nullptr, nullptr, nullptr};
  float2* e3[3] = {nullptr, nullptr, nullptr};
  float2* g2[3] = {nullptr, nullptr, nullptr};
  float2* g3[3] = {nullptr, nullptr, nullptr};
  float2* e1[3] = {nullptr, nullptr, nullptr};  // [slot][k], no 1/N
  long long e2s[3], e3s[3], e1s[3];
  int n_slots = 0;
  bool any_flip[3] = {false, false, false};
  std::vector<int> flip_slots[3];
  int* d_flip_slots[3] = {nullptr, nullptr, nullptr};
  // Phase seeds (null when some axis has no pipelined kernel or a
  // non-linear kGrid): sd2[m] / sd3[m] for the e2 / e3 passes of rotation m,
  // sd2t for the last e2 pass with et{1}{2} fused, sd1[a] for the
  // translation passes. Strides are elements per slot, widths per row.
  float2* sd2[3] = {nullptr, nullptr, nullptr};
  float2* sd3[3] = {nullptr, nullptr, nullptr};
  float2* sd1[3] = {nullptr, nullptr, nullptr};
  float2* sd2t = nullptr;
  long long sd2s[3] = {0, 0, 0}, sd3s[3] = {0, 0, 0}, sd1s[3] = {0, 0, 0}, sd2ts = 0;
  int sdw[3] = {0, 0, 0};  // row width of seeds along axis a (2*F1 + 2)
};

void dis_slot_params(const float* T, int n_states, const int* slots, int n_slots, int di,
                     std::vector<SlotParams>* out);
int dis_build_tables(disorder_ctx_s* ctx, const disorder_plan_s* plan, const std::vector<SlotParams>& sp,
                     bool with_grad, Workspace* ws, Tables* tb);
constexpr int kMaxStaticSlots = 256;
int dis_build_tables_into(disorder_ctx_s* ctx, const disorder_plan_s* plan, const SlotParams* sp, int ns,
                          char* base, size_t cap, Tables* tb);
// per-slot scalars into a caller array (no heap)
void dis_slot_params_into(const float* T, int n_states, int di, SlotParams* out);
// bytes dis_build_tables_into places in its region for ns slots
size_t dis_static_table_bytes(const disorder_plan_s* plan, int ns);
// device address of the static scratch of disorder_sinc_rigid_transform_static
// on the current device (noalloc.cu); called once when a context is created
int dis_static_scratch_resolve(void** addr, size_t* bytes);

// transform drivers (ops.cu)
int dis_forward_transform(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float2* x, long long x_s,
                          float2* z, const Tables& tb, int useFull, float2* yB /*3 vols per slot or null*/);
int dis_inverse_transform(disorder_ctx_s* ctx, const disorder_plan_s* plan, float2* u, const Tables& tb,
                          int useFull, float2* out, float beta /*accumulate when out!=null*/);

// ---------------------------------------------------------------- coil stage
struct CoilArgs {
  int N1, N2, N3c;         // N3c: readout length processed
  long long Vz;            // per-slot stride of z / u volumes
  const float2* Sf;        // coil maps, already offset to the first readout
  long long Sc;            // coil stride of Sf (full volume)
  int C;
  int n_slots;
  const int* d_slot_seg;   // segment of each slot
};

int dis_coil_expand_fft1(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a,
                         const float2* z, float2* A);
int dis_coil_fft2_gather(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a,
                         const float2* A, float2* y, long long y_ld, int y_n3off, int y_N3,
                         const float2* y_meas, float scale);
int dis_coil_scatter_ifft2(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a,
                           const float2* y, long long y_ld, int y_n3off, int y_N3, const float* We,
                           const float* Mb, float2* A);
int dis_coil_fft2_weight(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a, float2* A,
                         const float* wmap /*[seg][N1][N2], kz fastest*/,
                         float2* ys = nullptr, long long ys_ld = 0, int ys_n3off = 0, int ys_N3 = 0);
int dis_coil_ifft1_combine(disorder_ctx_s* ctx, const disorder_plan_s* plan, const CoilArgs& a,
                           const float2* A, float2* u, float scale);
int dis_build_weight_map(disorder_ctx_s* ctx, const disorder_plan_s* plan, const float* We, float* wmap,
                         float scale);

// ---------------------------------------------------------------- reductions / vector ops
int dis_seg_sums(disorder_ctx_s* ctx, const disorder_plan_s* plan, const int* d_slot_seg, int n_slots,
                 const float2* r, const float2* G /*nullable*/, long long G_stride, long long ld, int n3off, int N3c,
                 int N3full, int C, const float* wrow, double* d_out /*[n_slots][28]*/, Workspace* ws);


// tensor-core Gram of compressCoils (umma_gram.cu): partials part[b][c*C+d]
int dis_gram_umma(disorder_ctx_s* ctx, const float2* S, int C, long long V, float reg, double* part, int grid,
                  int mode);

// launch accounting
inline void dis_count(disorder_ctx_s* ctx, int n = 1) { ctx->launches += n; }

// CTAs of a kernel that fit on one SM of the current device by its registers,
// shared memory (with the largest carveout) and threads; 0 on error
int dis_ctas_per_sm(const void* fn, int threads, size_t dyn_smem);
