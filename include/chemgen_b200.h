/*
 * chemgen_b200: C ABI of the B200 getrates library (libchemgen_b200.so).
 *
 * getrates(P, T, Y) -> wdot: net molar production rate of every species at
 * every grid point, in the reference's units and layout:
 *   P     dyne/cm^2, double[ng]
 *   T     K,         double[ng]
 *   Y     mass fractions, double[ns*ng], species-major: Y[k*ng + i]
 *   wdot  mol/(cm^3 s),   double[ns*ng], same layout
 * (reference: chemgen/templates/reactions_hip/hip_v1_h.j2:7-13 and
 *  chemgen/templates/reactions_hip/device_functions_h.j2:701-719).
 *
 * Every call returns a chemgen_status; nothing here exits the process or
 * prints (the reference's HIP wrappers print and return, constants.py:7-24,
 * and its rocBLAS path exits, reactions_hip/hip_v4_h.j2:12-23).
 * Device-pointer calls are asynchronous on the given stream (NULL = the
 * legacy default stream); host-pointer calls return when wdot is on the host.
 */
#ifndef CHEMGEN_B200_H
#define CHEMGEN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum chemgen_status {
    CHEMGEN_OK = 0,
    CHEMGEN_ERR_INVALID_ARGUMENT = 1,   /* NULL handle/pointer, ng < 0, bad mode */
    CHEMGEN_ERR_BAD_MECHANISM = 2,      /* blob rejected by the parser */
    CHEMGEN_ERR_CUDA = 3,               /* a CUDA runtime call failed */
    CHEMGEN_ERR_OUT_OF_MEMORY = 4,
    CHEMGEN_ERR_MISALIGNED = 5,         /* a device pointer is not 8-byte aligned */
    CHEMGEN_ERR_UNSUPPORTED = 6,        /* mechanism outside what a path supports */
    CHEMGEN_ERR_TOO_LARGE = 7,          /* ng beyond a fixed capacity */
    CHEMGEN_ERR_NO_GLOBAL_MECHANISM = 8 /* drop-in wrapper called before chemgen_init_constants */
} chemgen_status;

/* Arithmetic modes of chemgen_getrates_ex. */
typedef enum chemgen_mode {
    CHEMGEN_MODE_FP64 = 0,              /* plain FP64, the reference's arithmetic */
    CHEMGEN_MODE_MIXED = 1              /* FP32 rate math, FP64 Gibbs/Kc exponents and wdot sums */
} chemgen_mode;

typedef struct chemgen_handle chemgen_handle;

const char* chemgen_version(void);
const char* chemgen_status_string(int status);

/* Load a packed mechanism (chemgen_b200/pack.py) onto `device`.
 * Replaces: copyConstantsToDevice (chemgen/constants.py:119-240) and
 * init_chemgen's allocations (chemgen/templates/chemgen_mod.j2:108-137).
 * Unlike the reference's __constant__ symbols, any number of handles coexist. */
int chemgen_create(const void* blob, size_t nbytes, int device, chemgen_handle** out);
int chemgen_destroy(chemgen_handle* h);
int chemgen_num_species(const chemgen_handle* h);
int chemgen_num_reactions(const chemgen_handle* h);

/* FP64 getrates on device pointers.
 * Replaces: getrates_hip_wrapper_v1..v4 (reactions_hip/hip_v1_cpp.j2:339-372,
 * hip_v2_cpp.j2:1078-1160) and the generated getrates (python_header.j2:25).
 * Any ng >= 0 (the reference requires ng to be a multiple of its block). */
int chemgen_getrates(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
                     double* wdot, void* stream);

/* Same with an explicit arithmetic mode. */
int chemgen_getrates_ex(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng,
                        const double* Y, double* wdot, void* stream);

/* FP64 getrates on the first min(*count, ng) points of arrays laid out for ng
 * points (species stride ng), with `count` a device pointer read by the
 * kernel (no counterpart in the reference).  For a batch whose size is known
 * only on the device, such as the points an error gate sends back
 * (chemgen_gate_select): a launch covers only the points counted, so the
 * batch can be sized for every point and nothing waits for the host.  Points
 * past the count are left as they are.  Runs on the staged FP64 kernel;
 * CHEMGEN_ERR_UNSUPPORTED for a mechanism too large for it.  Asynchronous. */
int chemgen_getrates_counted(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
                             double* wdot, const uint64_t* count, void* stream);

/* Scratch a call needs for `ng` points in `mode` (0 when the per-point state
 * fits in shared memory), and the variant that uses caller-owned scratch of
 * at least that many bytes (256-byte aligned) instead of library-owned memory. */
int chemgen_workspace_bytes(const chemgen_handle* h, int mode, int64_t ng, size_t* bytes);
int chemgen_getrates_ws(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng,
                        const double* Y, double* wdot, void* workspace, size_t workspace_bytes, void* stream);

/* Host-pointer getrates: copies P, T, Y to the device, computes, copies wdot
 * back, and returns when wdot is on the host.  The copies of one chunk of
 * points overlap the kernels and copies of the others (three streams).  Pinned
 * host memory gives the fastest copies; pageable memory works.
 * Replaces: chemgen_m::getrates_gpu (chemgen/templates/chemgen_mod.j2:139-166),
 * which maps host arrays with OpenMP target data. */
int chemgen_getrates_host(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng,
                          const double* Y, double* wdot);

/* Kernels generated for one mechanism (generate_chemistry.py --language cuda
 * emits them; the reference's counterpart is its per-mechanism generated
 * getrates, chemgen/chemistry.py:326-341).  A generated module calls
 * chemgen_register_kernels when it is loaded; every handle whose blob has the
 * same 64-bit FNV-1a fingerprint then runs the generated kernels instead of
 * the table-driven ones.  chemgen_use_generated(h, 0) forces the
 * table-driven kernels; chemgen_kernel_kind reports which kernel a mode
 * runs: 1 generated, 0 table-driven, -1 unavailable. */
typedef int (*chemgen_kernel_fn)(int mode, const double* P, const double* T, int64_t ng, const double* Y,
                                 double* wdot, void* stream);
int chemgen_register_kernels(uint64_t fingerprint, int ns, int nr, unsigned modes, chemgen_kernel_fn fn);
int chemgen_use_generated(chemgen_handle* h, int enable);
int chemgen_kernel_kind(chemgen_handle* h, int mode);

/* Analytic derivatives (no counterpart in the reference, whose torch
 * prototype chemgen/chemistry_nn.py:15-85 never ran).
 * chemgen_jacobian: dense d wdot/d(T, Y) per point, J[(k*(ns+1) + c)*ng + i],
 *   column c = 0 for T, 1 + j for Y_j; precision 0 = double, 1 = float
 *   (FP64 rate evaluation and accumulation, J stored in FP32).  Each row is
 *   accumulated on chip and J is written once when a 32-point tile's state
 *   and two rows fit in shared memory (up to ~180 species); each tile's
 *   reaction derivatives or rate constants go to library-owned scratch of
 *   8*nr*32 doubles per SM (about 100 MB at 325 reactions).  Larger
 *   mechanisms accumulate J in place with library-owned scratch of 4*ns*ng
 *   doubles (FP32 accumulation for precision 1).
 * chemgen_getrates_vjp: given G = dL/dwdot [ns*ng], the adjoint
 *   gT = dL/dT [ng], gY = dL/dY [ns*ng] and (if gP != NULL) gP = dL/dP [ng],
 *   without forming J: up to ~110 species with each 32-point tile's state in
 *   shared memory and a result that does not depend on scheduling, beyond
 *   that with library-owned scratch of 4*ns*ng doubles. */
int chemgen_jacobian(chemgen_handle* h, int precision, const double* P, const double* T, int64_t ng,
                     const double* Y, void* J, void* stream);
int chemgen_getrates_vjp(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
                         const double* G, double* gT, double* gY, double* gP, void* stream);

/* Learned surrogate of wdot (no counterpart in the reference; its torch
 * prototype chemgen/chemistry_nn.py:15-85 never ran).  Building blocks of a
 * BF16 MLP (FP32 accumulation) trained and evaluated on the GPU; all pointers
 * are device pointers, all calls asynchronous on `stream`.
 * chemgen_mlp_gemm: C[i*ldc + j] (+)= sum_r A[i*sai + r*sar] * B[j*sbj + r*sbr]
 *   for i < M, j < N, r < R (A, B BF16; C FP32; accumulate != 0 adds).
 * chemgen_mlp_bias_gelu: Z += bias (per column); H = GELU(Z) (tanh form) or Z, BF16.
 * chemgen_mlp_gelu_backward: dZ = dH * GELU'(Z) (BF16, and FP32 if dZf).
 * chemgen_mlp_mse_grad: loss += mean_rows sum_j colw_j (out - target)^2, dout = its gradient.
 * chemgen_mlp_colsum: db[n] = sum_m dZ[m*N + n].
 * chemgen_mlp_adam: Adam step (weight decay wd) on FP32 w, BF16 copy to wb (if non-NULL); the
 *   learning rate and bias corrections are read on the device from hyper = {lr, 1/(1-b1^t), 1/(1-b2^t)}.
 * chemgen_surrogate_features: per point the din values (1000/T, ln T, ln(P/1 atm), ln X_k for the
 *   ns species (mole fractions from Y and inv_mw; ln Y_k when inv_mw is NULL), zeros), each centred
 *   and scaled by the pairs in norm[0..7] (species values clipped to [-6, 6]); stored as BF16 hi
 *   parts in X[i*2*din + j] and BF16 remainders in X[i*2*din + din + j] (+FP32 in Xf if non-NULL).
 * chemgen_surrogate_targets: T[i*dout + k] = w_k / |w|_2 for k < ns, (ln |w|_2 - lnorm[0]) / lnorm[1]
 *   for k = ns, 0 beyond.
 * chemgen_surrogate_decode: the inverse, W[k*ng + i]; err_est[i] = column ns + 1. */
int chemgen_mlp_gemm(const void* A, int64_t sai, int64_t sar, const void* B, int64_t sbj, int64_t sbr, float* C,
                     int64_t ldc, int M, int N, int R, int accumulate, void* stream);
int chemgen_mlp_bias_gelu(float* Z, const float* bias, void* H, int64_t M, int N, int apply_gelu, void* stream);
int chemgen_mlp_gelu_backward(const float* dH, const float* Z, void* dZ, float* dZf, int64_t n, void* stream);
int chemgen_mlp_mse_grad(const float* out, const float* target, const float* colw, void* dout, float* doutf,
                         float* loss, int64_t M, int N, void* stream);
int chemgen_mlp_colsum(const float* dZ, float* db, int64_t M, int N, void* stream);
int chemgen_mlp_adam(float* w, const float* g, float* m, float* v, void* wb, int64_t n, const float* hyper, float b1,
                     float b2, float eps, float wd, void* stream);
int chemgen_surrogate_features(const double* P, const double* T, const double* Y, int64_t ng, int ns, int din,
                               const float* norm, const double* inv_mw, void* X, float* Xf, void* stream);
int chemgen_surrogate_targets(const double* W, int64_t ng, int ns, int dout, const float* lnorm, float* Tg,
                              void* stream);
int chemgen_surrogate_decode(const float* out, int64_t ng, int ns, int dout, const float* lnorm, double* W,
                             float* err_est, void* stream);

/* Fused surrogate inference on the tensor cores (no counterpart in the
 * reference): features, the four layers (tcgen05.mma, activations kept in
 * shared and tensor memory) and the decode to FP64 wdot in one kernel, for the
 * network above with din = 64, hidden 256, dout = 64 and ns <= 61.
 * chemgen_surrogate_pack: W1 [256 x 64], W2, W3 [256 x 256], W4 [64 x 256] (BF16, row-major
 *   [out x in]) -> img (chemgen_surrogate_image_elems() BF16 elements, 16-byte aligned), the
 *   operands in the tensor cores' K-major canonical layout, layer 1 with its input weights twice.
 * chemgen_surrogate_infer: wdot[k*ng + i] and err_est[i] (may be NULL) from (P, T, Y) with bias =
 *   (b1, b2, b3 [256 each], b4 [64]), norm[8], lnorm[2] and inv_mw[ns] as in
 *   chemgen_surrogate_features / _decode.  range (device, may be NULL) = {T_lo, T_hi, P_lo, P_hi}:
 *   a point with T or P outside it, a negative Y_k, |sum Y - 1| >= 1e-6 or a NaN gets
 *   err_est = +inf, so that an error gate sends it to the exact kernel.  Asynchronous on `stream`.
 * chemgen_surrogate_infer_error: 1 if a bounded wait inside the kernel ever gave up (its outputs
 *   are then incomplete), 0 otherwise, -1 on a CUDA error; synchronous; reset != 0 clears it. */
/* Training products on the tensor cores (tcgen05), each fused with what
 * follows it (no counterpart in the reference).  chemgen_mlp_gemm_tc:
 *   acc[m][n] = sum_k A[m*lda + k] B[n*ldb + k] (A [M x K], B [N x K], BF16,
 *   K-major, 16-byte aligned, lda and ldb multiples of 8; M a multiple of 128,
 *   N one of 32, 64 or a multiple of 128, K a multiple of 64), then epilogue
 *   0 STORE          C[m*ldc + n] (+)= acc (accumulate != 0 adds)
 *   1 STORE_T        C[n*ldc + m] (+)= acc
 *   2 BIAS_GELU      z = acc + bias[n]; C = z (if C); H[m*ldh + n] and HT[n*ldt + m] = GELU(z) (BF16, if given)
 *   3 BIAS           z = acc + bias[n]; C = z; H, HT = z (if given)
 *   4 GELU_BACKWARD  d = acc * GELU'(zprev[m*ldz + n]); C = d (if C); H, HT = d (BF16, if given)
 *   with GELU the tanh form of chemgen_mlp_bias_gelu.  C (except for STORE_T) and zprev: 16-byte
 *   aligned with ldc, ldz multiples of 4; H: 16-byte aligned with ldh a multiple of 8.
 *   Asynchronous on `stream`.
 * chemgen_mlp_tc_error: 1 if a bounded wait inside chemgen_mlp_gemm_tc gave
 *   up (outputs incomplete), else 0, -1 on a CUDA error; reset != 0 clears it.
 * chemgen_mlp_transpose_bf16: dst[c*ldd + r] = src[r*lds + c], r < rows, c < cols.
 * chemgen_mlp_adam_multi: one Adam step (as chemgen_mlp_adam) over `count` <= 8 FP32 tensors
 *   [rows[k] x cols[k]] in one launch, with weight decay decay[k] (decay may be NULL: none); the
 *   host arrays hold device pointers.  Per tensor it also writes, where the pointer is not NULL,
 *   wb[k] = BF16(w), wt[k][c*rows + r] = BF16(w[r][c]) and wd[k][r*2cols + c] =
 *   wd[k][r*2cols + cols + c] = BF16(w[r][c]) (wb, wt, wd themselves may be NULL). */
int chemgen_mlp_gemm_tc(const void* A, int64_t lda, const void* B, int64_t ldb, int M, int N, int K, int epilogue,
                        const float* bias, const float* zprev, int64_t ldz, float* C, int64_t ldc, void* H,
                        int64_t ldh, void* HT, int64_t ldt, int accumulate, void* stream);
int chemgen_mlp_tc_error(int reset);
int chemgen_mlp_transpose_bf16(const void* src, int64_t lds, int rows, int cols, void* dst, int64_t ldd,
                               void* stream);
/* Fused training passes of the surrogate network (din -> 256 -> 256 -> 256 -> 64, GELU on the
 * hidden layers), one CTA per 128 batch rows, B a multiple of 128, all BF16 operands 16-byte
 * aligned.  chemgen_mlp_forward_tc: X [B x K0] (row stride ldx, a multiple of 8; K0 = 64, or
 *   128 for hi + lo parts with W[0] = the first layer's weights twice side by side), W[0..3]
 *   [N x K] BF16, b[0..3] FP32 -> ZT[l] = (H_{l-1} W_l^T + b_l)^T [256 x B] FP32, HT[l] =
 *   GELU(Z_l)^T [256 x B] BF16 (l < 3), out = H_2 W_3^T + b_3 [B x 64] FP32 (16-byte aligned).
 * chemgen_mlp_backward_tc: dout [B x 64] BF16, WT[1..3] = W_l^T [in x out] BF16 (WT[0] unused),
 *   ZT[0..2] from the forward -> dZT[l] = dZ_l^T [256 x B] BF16 with dZ_2 = (dout W_3) *
 *   GELU'(Z_2), dZ_1 = (dZ_2 W_2) * GELU'(Z_1), dZ_0 = (dZ_1 W_1) * GELU'(Z_0); gb[l][n] =
 *   sum_m dZ_l[m][n] (FP32, 256 each, overwritten, summed in a fixed order); doutT = dout^T
 *   [64 x B] BF16.  work: chemgen_mlp_backward_tc_work_bytes(B) bytes of device memory, 16-byte
 *   aligned, zeroed before its first use and left zeroed (one call at a time per buffer).
 * Both asynchronous on `stream`; a time-out of a bounded wait sets chemgen_mlp_tc_error. */
int chemgen_mlp_forward_tc(const void* X, int64_t ldx, int K0, const void* const* W, const float* const* b, int B,
                           float* const* ZT, void* const* HT, float* out, void* stream);
size_t chemgen_mlp_backward_tc_work_bytes(int B);
int chemgen_mlp_backward_tc(const void* dout, const void* const* WT, const float* const* ZT, int B,
                            void* const* dZT, float* const* gb, void* doutT, void* work, void* stream);
int chemgen_mlp_adam_multi(int count, float* const* w, const float* const* g, float* const* m, float* const* v,
                           void* const* wb, void* const* wt, void* const* wd, const int* rows, const int* cols,
                           const float* decay, const float* hyper, float b1, float b2, float eps, void* stream);

int chemgen_surrogate_image_elems(void);
int chemgen_surrogate_pack(const void* W1, const void* W2, const void* W3, const void* W4, void* img, void* stream);
int chemgen_surrogate_infer(const void* img, const float* bias, const float* norm, const float* lnorm,
                            const double* inv_mw, int ns, const double* P, const double* T, int64_t ng,
                            const double* Y, double* wdot, float* err_est, const double* range, void* stream);
int chemgen_surrogate_infer_error(int reset);

/* Per-point error gate of the surrogate on the device (no counterpart in the
 * reference): the points whose error estimate fails are gathered into a
 * compact batch for the exact kernel and its results scattered back, all
 * asynchronous on `stream`, so the host need not read the count between the
 * surrogate's kernel and the exact one.
 * chemgen_gate_select: *count = the number of points i < ng with !(est[i] <= thr) (NaN fails);
 *   the first min(*count, cap) of them get their index in idx[0, cap), in no fixed order.
 *   A count above cap leaves the rest unlisted: the caller reads *count afterwards and treats
 *   them itself.  *count is zeroed by the call.
 * chemgen_gate_gather: for j < min(*count, cap): Pc[j] = P[idx[j]], Tc[j] = T[idx[j]],
 *   Yc[k*cap + j] = Y[k*ng + idx[j]]; slots past the count are left as they are.
 * chemgen_gate_scatter: for j < min(*count, cap): W[k*ng + idx[j]] = Wc[k*cap + j].
 * Pointers are device pointers, 8-byte aligned. */
int chemgen_gate_select(const float* est, float thr, int64_t ng, int64_t* idx, int64_t cap, uint64_t* count,
                        void* stream);
int chemgen_gate_gather(const double* P, const double* T, const double* Y, int ns, int64_t ng, const int64_t* idx,
                        const uint64_t* count, int64_t cap, double* Pc, double* Tc, double* Yc, void* stream);
int chemgen_gate_scatter(const double* Wc, int ns, int64_t cap, const int64_t* idx, const uint64_t* count,
                         double* W, int64_t ng, void* stream);

/* FP64 getrates that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc while they run -- a
 * solver that owns the device memory pool or forbids allocation (and the
 * device synchronisation cudaMalloc/cudaFree can cause) inside its time-step
 * loop.  The per-point state that the large-mechanism FP64 kernel keeps in
 * scratch lives in a fixed 16 MiB device array inside the library instead of
 * a library allocation; a GPU holds it from the moment the array's module is
 * loaded there until exit.  Under CUDA's lazy module loading (the default)
 * that load can happen at this entry point's first call on a device, and then
 * allocates and may synchronise the device; that first call also looks up the
 * array's address (with that device current).  So make one call per device
 * during set-up, before any stream capture and outside any loop that must not
 * allocate.  Device pointers and layouts as chemgen_getrates.  A mechanism
 * whose state slice of 3*ns*64 doubles exceeds the array (ns > 10922) returns
 * CHEMGEN_ERR_TOO_LARGE.  All calls share the array, so calls that overlap on
 * the GPU race. */
int chemgen_getrates_noalloc(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
                             double* wdot, void* stream);

/* Drop-in for the reference's process-global API.
 * chemgen_init_constants replaces copyConstantsToDevice
 * (chemgen/constants.py:119-240): it installs one process-wide mechanism.
 * getrates_hip_wrapper_v1 has the exact signature of the reference's wrapper
 * (reactions_hip/hip_v1_h.j2:7-13): device pointers, ng points, Y/wdot
 * species-major, log_eg and log_c caller-owned scratch of ng*ns doubles each
 * (used here as the per-point state when the mechanism is too large for
 * shared memory), synchronous on the default stream.  It returns void like
 * the reference; chemgen_last_wrapper_status() reports the outcome. */
int chemgen_init_constants(const void* blob, size_t nbytes);
int chemgen_free_constants(void);
void getrates_hip_wrapper_v1(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c);
int chemgen_last_wrapper_status(void);

/* The reference's Fortran module chemgen_m picks one of four wrappers at
 * build time (chemgen/templates/chemgen_mod.j2:139-166): v2, the fused
 * shared-memory kernel (reactions_hip/hip_v2_cpp.j2:1078-1160), v3, the
 * species-split reduction (hip_v3_cpp.j2:1144), and v4, the rocBLAS
 * formulation (hip_v4_cpp.j2:422, declared in hip_v4_h.j2:26-32).  All four
 * keep v1's signature and meaning, and here all four run the same kernels:
 * whichever the solver was built against links. */
void getrates_hip_wrapper_v2(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c);
void getrates_hip_wrapper_v3(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c);
void getrates_hip_wrapper_v4(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c);

/* Replaces allocate_intermediate_DeviceMemory (chemgen/constants.py:435-470),
 * which chemgen_m::init_chemgen calls for v4: here it reserves the
 * library-owned scratch that FP64 calls of up to ng points on the
 * process-wide mechanism need (none when the state fits in shared memory), so
 * that later wrapper calls do not allocate.  Returns void like the reference;
 * chemgen_last_wrapper_status() reports the outcome. */
void allocate_intermediate_DeviceMemory(int ng);

/* chemgen_init_constants from a blob file (generate_chemistry.py writes it
 * beside the kernels): path, or when path is NULL or empty the file named by
 * the environment variable CHEMGEN_BLOB, else "getrates.blob" in the working
 * directory.  For callers such as Fortran init_chemgen(flag, ng) whose
 * signature names no mechanism (chemgen/templates/chemgen_mod.j2:108-137). */
int chemgen_init_constants_file(const char* path);

/* Species count of the process-wide mechanism (-1 before
 * chemgen_init_constants): what chemgen_m sizes its EG and C scratch with,
 * where the reference's generated module has it as a constant
 * (chemgen/templates/chemgen_mod.j2:118-120). */
int chemgen_global_num_species(void);

#ifdef __cplusplus
}
#endif

#endif /* CHEMGEN_B200_H */
