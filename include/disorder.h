/*
 * libdisorder: B200-native (sm_100a) aligned-reconstruction hot path of
 * DISORDER (motion-corrected 3-D MRI). C ABI: plain pointers and sizes, no
 * framework types.
 *
 * Conventions (all follow the reference MATLAB code, column-major):
 *  - complex data are interleaved single precision (re, im) pairs;
 *  - a volume x is N1 x N2 x N3 with dims 1-2 the phase encodes (ky, kz) and
 *    dim 3 the readout; element (n1,n2,n3) is at n1 + N1*(n2 + N2*n3);
 *  - coil sensitivities Sf are N1 x N2 x N3 x C (coil slowest);
 *  - motion states are the slowest dim of a batch of volumes (dim 5);
 *  - samples y are Ns x 1 x N3 x C (sample fastest, then readout, then coil),
 *    grouped by segment as in Methods/buildHarmonicSampling.m;
 *  - rigid transforms T are n_states x 6, parameter-major (T[p*n + s]), the
 *    reference's [1 1 1 1 NS 6] array: translations t1..t3 in voxels of the
 *    full-resolution grid, then rotations r1..r3 in radians;
 *  - "device" pointers are CUDA device memory of the context's device;
 *    "host" pointers are ordinary host memory.
 * Every entry point returns a disorder_status; disorder_last_error() gives
 * the message of the last failure on a context. Calls are stream-ordered on
 * the context's stream and return after the work is enqueued unless noted;
 * entry points with host outputs synchronise the stream.
 */
#ifndef DISORDER_H
#define DISORDER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DISORDER_OK = 0,
  DISORDER_BAD_ARG = 1,
  DISORDER_UNSUPPORTED_FIELD = 2,
  DISORDER_OOM = 3,
  DISORDER_CUDA_ERR = 4,
  DISORDER_TIMEOUT = 5,
  DISORDER_NONFINITE = 6
} disorder_status;

typedef struct disorder_ctx_s* disorder_ctx;
typedef struct disorder_plan_s* disorder_plan;

/* ---- context, stream and memory (replaces MATLAB gpuArray/gather,
 *      Methods/fftGPU.m:27-31 device selection; the MEX handle layer) ---- */
int disorder_ctx_create(int device, disorder_ctx* out);
/* Plans, networks and device memory of a context are released before it:
 * disorder_plan_destroy, disorder_net_destroy and disorder_free use the
 * context's stream. */
int disorder_ctx_destroy(disorder_ctx ctx);
const char* disorder_last_error(disorder_ctx ctx);
int disorder_ctx_set_stream(disorder_ctx ctx, void* cuda_stream); /* NULL: own stream */
void* disorder_ctx_get_stream(disorder_ctx ctx);
int disorder_synchronize(disorder_ctx ctx);
/* Device memory from the device's stream-ordered pool: usable by work on the
 * context's stream at once, and by host code after disorder_synchronize.
 * disorder_free returns it in stream order without waiting; the pool keeps
 * freed memory for reuse until the process exits. */
int disorder_malloc(disorder_ctx ctx, size_t bytes, void** dptr);
int disorder_free(disorder_ctx ctx, void* dptr);
int disorder_memcpy_h2d(disorder_ctx ctx, void* dst, const void* src, size_t bytes);
int disorder_memcpy_d2h(disorder_ctx ctx, void* dst, const void* src, size_t bytes);
int disorder_memcpy_d2d(disorder_ctx ctx, void* dst, const void* src, size_t bytes);
/* The MEX gateway's 'upload' / gather pair: disorder_upload allocates bytes
 * (as disorder_malloc) and copies host data there, returning the device
 * pointer that stays resident behind a handle; disorder_download copies it
 * back to host memory. Free with disorder_free. */
int disorder_upload(disorder_ctx ctx, const void* host, size_t bytes, void** dptr);
int disorder_download(disorder_ctx ctx, const void* dptr, void* host, size_t bytes);
int disorder_memset(disorder_ctx ctx, void* dst, int value, size_t bytes);
/* number of kernels this context has launched since creation */
int64_t disorder_kernel_launches(disorder_ctx ctx);
/* Failure-path testing (no reference counterpart): arm one fault on the
 * context, taken by the next operation that reaches it and then cleared.
 * DISORDER_FAULT_TMA_WAIT: the next TMA line pass issues no tile loads, so
 *   its bounded tile waits run out (after a few milliseconds) with nothing in
 *   flight; the pass stops early and the next disorder_synchronize returns
 *   DISORDER_TIMEOUT. The context stays usable.
 * DISORDER_FAULT_OOM: the next workspace growth fails as a failed cudaMalloc
 *   would, and the call returns DISORDER_OOM. */
typedef enum {
  DISORDER_FAULT_NONE = 0,
  DISORDER_FAULT_TMA_WAIT = 1,
  DISORDER_FAULT_OOM = 2
} disorder_fault;
int disorder_ctx_inject_fault(disorder_ctx ctx, int32_t fault);
/* Arithmetic of the contractions that can run on the tensor cores (no
 * reference counterpart; the reference computes them in single precision):
 * DISORDER_PRECISION_FP32 (default): FP32 on the CUDA cores.
 * DISORDER_PRECISION_BF16X3: tcgen05 MMAs on operands split into two BF16
 *   parts, hi*hi + hi*lo + lo*hi accumulated in FP32 (about 16 significant
 *   bits per operand).
 * DISORDER_PRECISION_TF32X3: the same with two TF32 parts (about 21 bits).
 * The setting applies to the coil-compression Gram matrix
 * (disorder_compress_coils) and to the DFT line passes of the sinc rigid
 * transform that have a tensor-core kernel. */
typedef enum {
  DISORDER_PRECISION_FP32 = 0,
  DISORDER_PRECISION_BF16X3 = 1,
  DISORDER_PRECISION_TF32X3 = 2
} disorder_precision;
int disorder_ctx_set_precision(disorder_ctx ctx, int32_t mode);
/* Kernel choices of one context, set by an autotuner (no reference
 * counterpart). DISORDER_TUNE_TMA: 1 (default) moves the tiles of the strided
 * line passes with TMA bulk tensor copies, 0 with per-thread cp.async
 * pipelines (same results). DISORDER_TUNE_COIL_STAGE: 0 (default) runs the
 * encoding operators' coil stage as three passes over per-coil volumes, 1 as
 * per-tile sample sums without them (same results to rounding; new contexts
 * start at 1 when the environment sets DISORDER_SUM_COIL=1). */
typedef enum { DISORDER_TUNE_TMA = 0, DISORDER_TUNE_COIL_STAGE = 1 } disorder_tune_key;
int disorder_ctx_set_tuning(disorder_ctx ctx, int32_t key, int32_t value);
/* bytes of device workspace the context holds (operator, solver and reduction
 * buffers it grows on demand and keeps until disorder_ctx_destroy); a
 * diagnostic with no reference counterpart */
int64_t disorder_workspace_bytes(disorder_ctx ctx);
/* CUDA-event timing on the context's stream (no reference counterpart):
 * disorder_event_record(ctx, slot) records event `slot` (0..15);
 * disorder_event_elapsed(ctx, a, b, &ms) synchronises on b and returns the
 * device time between the two events in milliseconds. */
int disorder_event_record(disorder_ctx ctx, int32_t slot);
int disorder_event_elapsed(disorder_ctx ctx, int32_t a, int32_t b, float* ms);

/* ---- plan: the geometry and sampling fields of the E structure ----
 * Replaces generateTransformGrids (Methods/generateTransformGrids.m:23-67:
 * E.kG, E.rkG) and the sample bookkeeping of buildHarmonicSampling
 * (Methods/buildHarmonicSampling.m:25-50: E.Fs as DFT-row indices, E.nEc). */
typedef struct {
  int32_t N[3];        /* grid size at this level */
  const float* rG[3];  /* host: rGrid{m}, N[m] values (full-res voxel units) */
  const float* kG[3];  /* host: kGrid{m}, ifftshifted (sh=1), N[m] values */
  float cent[3];       /* host: flip centre per dim (cGrid, default N/2+1) */
} disorder_grid_desc;

typedef struct {
  int32_t n_seg;              /* E.NSe: segments (motion states + outer) */
  int32_t n_mot;              /* E.NMs: leading segments with a transform */
  const int64_t* seg_offsets; /* host: E.nEc, n_seg+1 sample offsets */
  const int32_t* ky;          /* host: 0-based DFT row of dim 1 per sample */
  const int32_t* kz;          /* host: 0-based DFT row of dim 2 per sample */
} disorder_sampling_desc;

int disorder_plan_create(disorder_ctx ctx, const disorder_grid_desc* grid,
                         const disorder_sampling_desc* smp, disorder_plan* out);
int disorder_plan_destroy(disorder_plan plan);

/* ---- sinc rigid transform ----
 * [x,xB]=sincRigidTransform(x,et,di,F,FH,sumR,useFull) with et from
 * precomputeFactorsSincRigidTransform(kG,rkG,T,di,0,1,1)
 * (Methods/sincRigidTransform.m:1-116; Methods/precomputeFactorsSincRigidTransform.m:24-133).
 * x: device, x_states (1 or n_states) volumes. T: host n_states x 6.
 * di=1 forward: out holds n_states volumes. di=0 inverse: out holds the sum
 * over states when sumR!=0, else n_states volumes. useFull: 1 full, 0
 * translations only, -1 rotations only. */
int disorder_sinc_rigid_transform(disorder_ctx ctx, disorder_plan plan, const void* x,
                                  int32_t x_states, const float* T, int32_t n_states,
                                  int32_t di, int32_t sumR, int32_t useFull, void* out);

/* et=precomputeFactorsSincRigidTransform(kG,rkG,T,di,0,1,1)
 * (Methods/precomputeFactorsSincRigidTransform.m:24-133, gr=1, sh=1) as device
 * arrays. The transforms above build these factors on the fly; this entry
 * point materialises them for callers that want the reference's et.
 * T: host n_states x 6. di: 1 forward, 0 inverse.
 * e1: 3 consecutive blocks, block m is N[m] x n_states: et{1}{m} =
 *     exp(i (-1)^di T(m) kGrid{m}) along dim m.
 * e2, e3: 3 consecutive blocks each, block m is N[a] x N[b] x n_states over
 *     the dims (a, b) = (1,2), (1,3), (2,3) for m = 1, 2, 3 that rkGrid{1}{m}
 *     and rkGrid{2}{m} span: et{2}{m} = exp((-1)^(di-1) i tan(theta_m/2)
 *     rkGrid{1}{m}) and et{3}{m} = exp((-1)^di i sin(theta_m) rkGrid{2}{m}),
 *     theta wrapped to +-pi/2 after the flip test (rkGrid in single precision,
 *     as the reference rounds it).
 * flip: host 3 x n_states, flip[m*n_states + s] = |theta_m| > pi/2 (et{5}{m}).
 * Any of e1, e2, e3, flip may be NULL. */
int disorder_precompute_factors(disorder_ctx ctx, disorder_plan plan, const float* T,
                                int32_t n_states, int32_t di, void* e1, void* e2, void* e3,
                                uint8_t* flip);

/* The sinc rigid transform above for callers that cannot let a library
 * allocate device memory (an application that reserves its whole device
 * budget at start-up and serves buffers from its own allocator, where a
 * cudaMalloc can fail and synchronises the device). No counterpart in the
 * reference. It allocates nothing: its scratch (the phase tables) lives in
 * one static 32 MiB device array that every GPU loading this library holds
 * until exit. Limits: at most 256 states and at most 32 MiB of tables per call
 * (about 12 states at 256x256x176, about 200 at 64x64x44), rotations within
 * +-90 degrees, and di=0 (inverse) takes n_states volumes and writes them
 * back without summing. Larger requests fail with DISORDER_BAD_ARG. The
 * array's device address is resolved when the context is created
 * (disorder_ctx_create, cudaGetSymbolAddress), which loads the module holding
 * it and commits its 32 MiB on that device then; the call itself allocates
 * nothing and loads no data module (its kernels, shared with the other
 * entry points, load on first use like any CUDA code unless
 * CUDA_MODULE_LOADING=EAGER). All calls share the one array and each call
 * rewrites the part it uses before reading it: calls that overlap on the GPU
 * (other streams, contexts or host threads) race with each other. The plan
 * must already exist (disorder_plan_create allocates). */
int disorder_sinc_rigid_transform_static(disorder_ctx ctx, disorder_plan plan, const void* x,
                                         int32_t x_states, const float* T, int32_t n_states,
                                         int32_t di, int32_t useFull, void* out);

/* G=sincRigidTransformGradient(xB,et,etg,F,FH)
 * (Methods/sincRigidTransformGradient.m:1-150) for the forward transform of
 * one volume x (device) by n_states transforms T (host). G: device, 6 x
 * n_states volumes, G[(g*n_states + s)*V]: derivatives with respect to
 * t1,t2,t3,r1,r2,r3. xT (device, optional): the transformed volumes. */
int disorder_sinc_rigid_transform_gradient(disorder_ctx ctx, disorder_plan plan,
                                           const void* x, const float* T, int32_t n_states,
                                           void* G, void* xT);

/* ---- encoding operators (Reconstruction/encode.m, decode.m, encodedecode.m) ----
 * Sf: device N1xN2xN3xC. T: host n_mot x 6 or NULL (no motion: the
 * reference's any(E.Tr(:)~=0) false branch). We: device per-sample weights
 * (EH.We) or NULL. Mb: device length-N3 readout weights (EH.Mb) or NULL. */
int disorder_encode(disorder_ctx ctx, disorder_plan plan, const void* x, const void* Sf,
                    int32_t n_coils, const float* T, void* y);
int disorder_decode(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                    int32_t n_coils, const float* T, const float* We, const float* Mb, void* x);
int disorder_encodedecode(disorder_ctx ctx, disorder_plan plan, const void* x, const void* Sf,
                          int32_t n_coils, const float* T, const float* We, void* out);

/* [En]=computeEnergy(y,x,E,R,EH) (Reconstruction/computeEnergy.m:34-80, no=2):
 * En[0] = sum |sqrt(Mb) sqrt(Mbe) (E x - y)|^2, En[1] = |sum Ti.*|x|^2|.
 * Mb, Mbe: device length-N3 or NULL. R_Ti: device real V or NULL. En: host. */
int disorder_compute_energy(disorder_ctx ctx, disorder_plan plan, const void* y, const void* x,
                            const void* Sf, int32_t n_coils, const float* T, const float* Mb,
                            const float* Mbe, const float* R_Ti, double* En);

/* ---- solvers ----
 * [x,En,~,~,nn]=CGsolver(y,E,EH,A,C,R,x,nIt,tolType,tol) with E.Je=1
 * (Reconstruction/CGsolver.m:1-119). tolType: 1 'RelativeResidual2Error',
 * 6 'Energy', 7 'None' (Reconstruction/stopCondition.m:10-21).
 * P_Se (A.Se), C_Ma (C.Ma), R_Ti (R.Ti.la): device real V arrays or NULL.
 * x_inout: device; used as the initial guess when x_init!=0, else x=0.
 * En: host, 2 x ceil(nIt/2) doubles (column-major), filled for tolType 6;
 * n_en, nn: host outputs (energy columns written, iterations run). */
int disorder_cg_solve(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                      int32_t n_coils, const float* T, const float* We, const float* Mb,
                      const float* Mbe, const float* P_Se, const float* C_Ma, const float* R_Ti,
                      void* x_inout, int32_t x_init, int32_t nIt, int32_t tolType, double tol,
                      double* En, int32_t* n_en, int32_t* nn);

/* disorder_cg_solve that also returns the final sample residual
 * r_out = encode(x) - y (device, samples x N3 x C, encode's layout). CG keeps
 * that residual beside its vectors, so the caller gets it without another
 * encode; solveXT.m:443 needs it after every image update at the outlier
 * levels. No separate reference function. */
int disorder_cg_solve_residual(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                               int32_t n_coils, const float* T, const float* We, const float* Mb,
                               const float* Mbe, const float* P_Se, const float* C_Ma,
                               const float* R_Ti, void* x_inout, int32_t x_init, int32_t nIt,
                               int32_t tolType, double tol, double* En, int32_t* n_en, int32_t* nn,
                               void* r_out);

/* E=LMsolver(y,E,x,C) (Reconstruction/LMsolver.m:1-226), E.Fs branch, one
 * Levenberg-Marquardt iteration over the motion states.
 * y: device samples (all segments, full readout). Sf: device.
 * x: device volume. T (E.Tr), w (E.w), cT (E.cT): host, updated in place.
 * winit, tL[2]: E.winit, E.tL. n3_lo/n3_hi: E.nF as the readout range
 * [n3_lo, n3_hi) (n3_hi<=0: whole readout). En, EnPrev: host n_mot doubles
 * (energy after/before, per state; E.En = min of the two). */
int disorder_lm_step(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                     int32_t n_coils, const void* x, float* T, float* w, uint8_t* cT,
                     float winit, const float* tL, int32_t n3_lo, int32_t n3_hi, double* En,
                     double* EnPrev);

/* ---- data preparation ----
 * x=resampling(x,Nres) for image-space complex data (Methods/resampling.m:45-94,
 * fo=0, no mirroring): per changed dim, DFT/Nin, centred crop or zero-pad,
 * inverse DFT*Nout. x, out: device, n_vols volumes of Nin / Nout. */
int disorder_resample(disorder_ctx ctx, const void* x, const int32_t* Nin, int32_t n_vols,
                      const int32_t* Nout, void* out);

/* Rows of a sample array picked for a pyramid level (the k-space crop of
 * Methods/downsampleOperators.m:48-51 on per-sample data):
 * y_out[i + n_out*r] = scale * y_in[idx[i] + n_in*r], r < rows (readout x coils).
 * idx: device int32 n_out. */
int disorder_gather_samples(disorder_ctx ctx, const void* y_in, int64_t n_in, int64_t rows,
                            const int32_t* idx, int64_t n_out, float scale, void* y_out);

/* A.Se = 1 ./ (sum_c |S_c|^2 + reg) (Reconstruction/solveXT.m:231-233,406-408):
 * Sf device V x C, out device real V. */
int disorder_precondition_weights(disorder_ctx ctx, const void* Sf, int32_t n_coils, int64_t V,
                                  float reg, float* out);

/* [S,y,C,D,U]=compressCoils(S,perc,y) (Methods/compressCoils.m:76-118, the
 * branch for equal coil and data grids): Gram matrix on the device, Hermitian
 * eigendecomposition on the host, compression on the device.
 * S: device V x C_in; y: device n_y x C_in or NULL; perc < 1: energy share,
 * >= 1: coil count; C_max > 0 caps the count. S_out (V x C_in capacity),
 * y_out (n_y x C_in capacity): device. C_out: host. D (C_in) and U
 * (C_in x C_in complex, interleaved, column-major): host or NULL. */
int disorder_compress_coils(disorder_ctx ctx, const void* S, int32_t C_in, int64_t V, const void* y,
                            int64_t n_y, double perc, int32_t C_max, void* S_out, void* y_out,
                            int32_t* C_out, double* D, double* U);

/* ---- per-state residuals (the quantities LMsolver.m:72,82-93 forms per state) ----
 * r = encode(T_s x) - y of every motion state s over the readout rows
 * [n3_lo, n3_hi) (n3_hi <= 0: all rows).
 * disorder_state_energies: En[s] = sum |r|^2 over state s's samples and
 *   those rows / numel(y), the normalisation of LMsolver.m:82-83. En: host n_mot.
 * disorder_backproject_states: out[s*V..] = T_s^H sum_c S_c^H F^H r_s, the
 *   adjoint of state s alone (no sum over states). out: device n_mot volumes. */
int disorder_state_energies(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                            int32_t n_coils, const void* x, const float* T, int32_t n3_lo,
                            int32_t n3_hi, double* En);
/* [Re]=computeEnergy(y,x,E,[],EH,[],[],[],[],1) (Reconstruction/computeEnergy.m:34-80,
 * no=2, avdi=1), the per-sample residual energies of the outlier weighting
 * (Reconstruction/solveXT.m:443): En[i] = sum over readout rows and coils of
 * Mbe[n3] |encode(x) - y|^2 for every sample i (all segments). Mbe: device
 * length N3 readout weights (EH.Mbe, or EH.Mb.*EH.Mbe when both are set) or
 * NULL (all ones). En: host n_samples doubles. */
int disorder_sample_energies(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                             int32_t n_coils, const void* x, const float* T, const float* Mbe,
                             double* En);
/* The same per-sample energies of a residual r that the caller already holds
 * (device, samples x N3 x C; for example from disorder_cg_solve_residual).
 * At most 2M samples. */
int disorder_residual_energies(disorder_ctx ctx, disorder_plan plan, const void* r, int32_t n_coils,
                               const float* Mbe, double* En);
int disorder_backproject_states(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                                int32_t n_coils, const void* x, const float* T, int32_t n3_lo,
                                int32_t n3_hi, void* out);

/* ---- synthetic scan data (the simulation recipe on the device) ----
 * The reference simulates acquisitions from a ground-truth image and coil
 * maps it loads from files (fig0506.m:53-56) and adds complex Gaussian noise
 * (Methods/plugNoise.m:17, Simulation/synthesizeY.m:82-84); these build the
 * stand-ins on the device. N: host int32[3]; out/S/y: device.
 * disorder_synth_phantom: out[v] = (sum over ellipsoids containing v of
 *   their magnitude) * exp(i sum_q a_q cos(2 pi f_q . r + p0_q)), r the grid
 *   coordinate -0.5 + i/N per axis. ell: host n_ell x 16 floats {centre[3],
 *   semi-axes[3], rotation R (row-major 3x3), magnitude}, a point is inside
 *   when |R (r - centre) / semi-axes| <= 1; ph: host n_ph x 5 floats {f[3],
 *   p0, a}. normalise != 0 divides the volume by its L2 norm.
 * disorder_synth_coils: S[v + c V] = g_c(v) exp(i phi_c(v)) / rss(v) with
 *   g_c = exp(-|r - centre_c|^2 / (2 width^2)), phi_c = 2 pi k_c . r / 4 +
 *   phase0_c, rss the root sum of squares of the g_c. cp: host C x 7 floats
 *   {centre[3], k[3], phase0}.
 * disorder_add_noise: y[e] += sigma (n1 + i n2), n1 and n2 standard normals
 *   that depend only on (seed, e). */
int disorder_synth_phantom(disorder_ctx ctx, const int32_t* N, int32_t n_ell, const float* ell, int32_t n_ph,
                           const float* ph, int32_t normalise, void* out);
int disorder_synth_coils(disorder_ctx ctx, const int32_t* N, int32_t C, const float* cp, float width, void* S);
int disorder_add_noise(disorder_ctx ctx, void* y, int64_t n, float sigma, uint64_t seed);

/* ---- learned motion proposal (no counterpart in the reference) ----
 * A 3-D convolutional network maps one state's back-projected residual and
 * the current image (two complex volumes read as 4 channels: residual real
 * and imaginary, image real and imaginary) to a 6-parameter motion update:
 * 4 convolutions 3x3x3, stride 2, zero padding 1, with 16, 32,
 * 64 and 64 output channels and GELU, a global average pool, and a
 * 64 -> 128 (GELU) -> 6 perceptron. Weights are BF16 on the device (FP32
 * master copy for training); activations and sums are FP32.
 * Parameters, in this order (flat FP32): per convolution l the weights
 * [tap = (kz*3 + ky)*3 + kx][c_in][c_out] and the bias [c_out]; then fc1
 * [64][128] and its bias [128]; then fc2 [128][6] and its bias [6].
 * Outputs 0-2 are translation updates / 2 in voxels of the input volume's
 * grid and outputs 3-5 rotation updates / 8 degrees.
 * D: input volume size (n1, n2, n3); max_batch: most volumes per call. */
typedef struct disorder_net_s* disorder_net;
/* ---- sample orders (Acquisition/samplingDISORDER.m) ----
 * The order in which samplingDISORDER.m:104 distributes a tile's n1 x n2
 * positions over consecutive segments: Acquisition/
 * electrostaticRepulsionDISORDER.m:9-52 (greedy minimum wrapped electric
 * repulsion, first minimum by more than 1e-9 in column-major scan order).
 * order: n1*n2 0-based column-major positions. Host computation; no context. */
int disorder_electrostatic_order(int32_t n1, int32_t n2, int32_t* order);

int64_t disorder_net_param_count(void);
int disorder_net_create(disorder_ctx ctx, const int32_t* D, int32_t max_batch, disorder_net* net);
int disorder_net_destroy(disorder_net net);
/* params: host FP32, disorder_net_param_count() values. */
int disorder_net_set_params(disorder_ctx ctx, disorder_net net, const float* params);
int disorder_net_get_params(disorder_ctx ctx, disorder_net net, float* params);
/* in: device, batch complex volumes of size D (channels 0-1), multiplied by
 * in_scale on read; ref: device, one complex volume shared by the batch
 * (channels 2-3), multiplied by ref_scale, or NULL for zeros. Both must stay
 * allocated until the backward of this forward. out: device batch x 6
 * (row-major), or NULL to keep it internal. */
int disorder_net_forward(disorder_ctx ctx, disorder_net net, const void* in, const void* ref,
                         int32_t batch, float in_scale, float ref_scale, float* out);
/* Gradient of loss = sum_b sum_k (out[b][k] - target[b][k])^2 / batch for the
 * inputs of the last disorder_net_forward. target: device batch x 6.
 * grad: device, param_count FP32 values (overwritten). loss: host. */
int disorder_net_backward(disorder_ctx ctx, disorder_net net, const float* target, int32_t batch,
                          float* grad, double* loss);
/* One Adam step on the FP32 master parameters with grad (device), then the
 * BF16 copies are refreshed. step: 1-based step count (bias correction). */
int disorder_net_adam(disorder_ctx ctx, disorder_net net, const float* grad, float lr, float beta1,
                      float beta2, float eps, int32_t step);
/* Proposed motion update of every motion state: back-project the states'
 * residuals at (x, T) over readout rows [n3_lo, n3_hi), run the network on
 * them (scaled by gain / rms(x)) with x (scaled by 1 / rms(x)) and convert
 * its outputs to T units
 * (translations scaled by the plan's grid spacing rG[m][1] - rG[m][0], the
 * full-grid voxels per volume voxel; rotations in radians).
 * dT: host n_mot x 6, parameter-major like T (dT[p*n_mot + s]). The plan's
 * volume size must equal the network's D. */
int disorder_propose_motion(disorder_ctx ctx, disorder_plan plan, disorder_net net, const void* y,
                            const void* Sf, int32_t n_coils, const void* x, const float* T,
                            int32_t n3_lo, int32_t n3_hi, float gain, float* dT);

/* ---- compressed-sensing reconstruction (Reconstruction/CSsolver.m) ----
 * A shearlet system (Shearlets/buildShearlet.m, 3-D, complex=0) held as its
 * 2-D planes: pair 0 = dims (1,2), pair 1 = dims (1,3), pair 2 = dims (3,2);
 * 3-D shearlet w is plane table[4w+1] of pair table[4w] times plane
 * table[4w+3] of pair table[4w+2] (buildShearlet.m:136-146). planesQ: host
 * complex64, n_planes planes of N[a] x N[b] (column-major, a = first dim of
 * the pair), frequency 0 first. Every N[m] must be a product of 2, 3, 5, 7,
 * 11 and 13 (else DISORDER_UNSUPPORTED_FIELD). */
typedef struct disorder_shearlet_s* disorder_shearlet;
int disorder_shearlet_create(disorder_ctx ctx, const int32_t N[3], int32_t n_planes, const void* planes0,
                             const void* planes1, const void* planes2, int32_t n_filters,
                             const int32_t* table, disorder_shearlet* sh);
int disorder_shearlet_destroy(disorder_shearlet sh);
/* computeShearlet (CSsolver.m:91-101) and R.Sh.We=(R.Sh.We+eps).^pw
 * (:59,80): We[w*V+v] = (|IDFT3(conj(S_w).*DFT3(x))|(v) + eps)^pw, with the
 * unnormalised DFT of fftGPU and the 1/N inverse of ifftGPU. x: device V
 * complex; We: device V x n_filters floats. */
int disorder_shearlet_coefficients(disorder_ctx ctx, disorder_shearlet sh, const void* x, float eps,
                                   float pw, float* We);
/* Shearlet branch of regularize.m:27-46: out = beta*out + scale *
 * IDFT3(sum_w S_w .* DFT3(We_w .* IDFT3(conj(S_w) .* DFT3(x)))), with
 * scale = R.Sh.la*R.Sh.p/2. x, out: device V complex (out may not alias x). */
int disorder_shearlet_regularize(disorder_ctx ctx, disorder_shearlet sh, const void* x, const float* We,
                                 float scale, float beta, void* out);
/* Regularizer term of traceEstimation.m:85-102 for one real probe:
 * tr = sum_w ||sqrt(We_w) .* IDFT3(conj(S_w) .* DFT3(probe))||^2 (host). */
int disorder_shearlet_trace(disorder_ctx ctx, disorder_shearlet sh, const float* probe, const float* We,
                            double* tr);
/* A probe of traceEstimation.m:54-59 on the device: V standard normals that
 * depend only on (seed, index) (plugNoise(x,1)), scaled to unit mean square,
 * times mask (C.Ma, device real V) when given. probe: device V floats. */
int disorder_trace_probe(disorder_ctx ctx, int64_t V, uint64_t seed, const float* mask, float* probe);
/* Fidelity term of traceEstimation.m:61-84 for one real probe:
 * tr = sum_c sum_k W(k1,k2) |F2(S_c .* probe)(k)|^2, F2 the unitary DFT over
 * dims 1-2 (fftGPU/sqrt(N)); W: device N1 x N2 weights (EH.We on the grid).
 * Sf: device V x C complex. N1 and N2 as for shearlet_create. */
int disorder_fidelity_trace(disorder_ctx ctx, const int32_t N[3], const float* probe, const void* Sf,
                            int32_t C, const float* wgrid, double* tr);
/* disorder_cg_solve with the shearlet term in the normal operator
 * (CSsolver.m:76, CGsolver.m:55,80 calling regularize.m:27-46):
 * EHE = constrain(encodedecode(p) + Ti.*p + scale*Sh(p; We)). */
int disorder_cg_solve_shearlet(disorder_ctx ctx, disorder_plan plan, const void* y, const void* Sf,
                               int32_t n_coils, const float* T, const float* We, const float* Mb,
                               const float* Mbe, const float* P_Se, const float* C_Ma,
                               const float* R_Ti, disorder_shearlet sh, const float* sh_We,
                               float sh_scale, void* x_inout, int32_t x_init, int32_t nIt,
                               int32_t tolType, double tol, double* En, int32_t* n_en, int32_t* nn);

#ifdef __cplusplus
}
#endif
#endif /* DISORDER_H */
