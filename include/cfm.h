/*
 * cfm.h -- C ABI of libcfm.so, the single-GPU (B200, sm_100a) CPU-free
 * iterative-solver library: Jacobi 2d5p / 3d7p sweeps and conjugate
 * gradient, each run as one persistent kernel that loops on the device
 * behind grid barriers.
 *
 * Conventions
 *  - Every entry point returns a cfm_status (int); no entry point exits the
 *    process.  cfm_last_error() gives a one-line description of the last
 *    failure seen by the calling thread.
 *  - Grids are row-major with x fastest: a[(z * ny + y) * nx + x].
 *    Cells x = 0 and x = nx-1 are fixed (Dirichlet) columns/faces.
 *    Rows y = 0, ny-1 (2D) and planes z = 0, nz-1 (3D) are periodic halo
 *    copies of rows ny-2, 1 (planes nz-2, 1), exactly as the reference's
 *    single-GPU run copies them after every sweep.
 *  - Host buffers passed in are owned by the caller.  Device buffers are
 *    owned by the library handle unless an entry point says otherwise.
 *  - Calls on one handle must come from one thread at a time.  Each handle
 *    issues all its work on one CUDA stream (its own, or the one set with
 *    the *_set_stream call).
 *
 * Reference interfaces these replace (paths within ParCoreLab/CPU-Free-model):
 *  - Stencil version table entry `int init(int argc, char **argv)`
 *      Stencil/jacobi2D/include/common.h:20, Stencil/jacobi3D/src/main.cu:31-53
 *  - single-GPU oracle `double single_gpu(nx, ny, iter_max, real *a_ref_h, ...)`
 *      Stencil/jacobi2D/src/common.cu:154-273, Stencil/jacobi3D/src/common.cu:110-239
 *  - CG version table entry `initfunc_t(int *dRowPtr, int *dCol, real *dVal,
 *      int n, int nnz, bool zero_indexed, int iter_max, real *x_final, ...)`
 *      CG/include/common.h:122-127
 */
#ifndef CFM_H
#define CFM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFM_API_VERSION 1

typedef enum cfm_status {
    CFM_OK = 0,
    CFM_BAD_ARG = 1,          /* invalid sizes, null pointers, unknown enum value */
    CFM_CUDA_ERROR = 2,       /* a CUDA runtime call failed (see cfm_last_error) */
    CFM_BARRIER_TIMEOUT = 3,  /* a device grid barrier wait ran out of its time budget */
    CFM_BREAKDOWN = 4,        /* CG: non-finite or non-positive curvature (alpha/beta) */
    CFM_NOT_CONVERGED = 5,    /* CG: iteration cap reached before the tolerance */
    CFM_NO_DEVICE = 6,        /* no CUDA device visible */
    CFM_UNSUPPORTED = 7,      /* request not supported by this build (e.g. grid too large) */
    CFM_OUT_OF_MEMORY = 8     /* device allocation failed */
} cfm_status;

typedef enum cfm_precision { CFM_FP64 = 0, CFM_FP32 = 1 } cfm_precision;

/* Initial-state generators.
 * CFM_PROBLEM_REF: the reference's own initial grid (2D: x columns at
 *   sin(2*pi*y/(ny-1)); 3D: x=0 face at z - y - (nx-1), x=nx-1 face 0,
 *   Stencil/jacobi3D/src/common.cu:15-29).
 * CFM_PROBLEM_CONFIG: 2D as REF; 3D both x faces at
 *   sin(2*pi*y/(ny-1)) * sin(2*pi*z/(nz-1)), periodic in y and z. */
typedef enum cfm_problem { CFM_PROBLEM_REF = 0, CFM_PROBLEM_CONFIG = 1 } cfm_problem;

/* Jacobi implementations, named for the reference version they stand in for
 * on one GPU. */
typedef enum cfm_jacobi_impl {
    /* "Baseline Copy": one kernel launch per sweep plus cudaMemcpyAsync halo
     * copies, host-controlled (Stencil/jacobi3D/src/baseline/multi-threaded-copy.cu) */
    CFM_JACOBI_HOST_LOOP = 0,
    /* "Baseline P2P": one launch per sweep, halos written by the kernel
     * (Stencil/jacobi3D/src/baseline/multi-threaded-p2p.cu) */
    CFM_JACOBI_HOST_LOOP_INKERNEL_HALO = 1,
    /* "Design 1"/"Design 2": CPU-free, one cooperative launch for all sweeps,
     * device grid barrier between sweeps (Stencil/jacobi2D/src/single-stream/
     * multi-threaded-two-block-comm.cu:9-105) */
    CFM_JACOBI_PERSISTENT = 2,
    /* "PERKS": CPU-free with each block's tile resident on chip across sweeps
     * (Stencil/jacobi2D/PERKS/jacobi-general-kernel.cuh:22-505) */
    CFM_JACOBI_RESIDENT = 3
} cfm_jacobi_impl;

typedef struct cfm_stats {
    double seconds;       /* device time of the solve, CUDA events on the handle's stream */
    long long iterations; /* sweeps (Jacobi) or CG iterations performed */
    double lups;          /* lattice-point updates (Jacobi) */
    double glups;         /* lups / seconds / 1e9 */
    double bytes;         /* algorithmic HBM bytes of the solve (16 B/LUP FP64, 8 FP32 for Jacobi) */
    double gbs;           /* bytes / seconds / 1e9 */
    double residual;      /* CG: final FP64 true relative residual ||b-Ax||/||b|| */
    double h2d_bytes;     /* host->device bytes copied inside the call */
    double d2h_bytes;     /* device->host bytes copied inside the call */
    int launches;         /* kernel launches issued inside the timed region */
    int status;           /* cfm_status of the run */
    int refinements;      /* mixed precision: FP64 reliable updates; standard / pipelined CG: restarts */
    int pad;
} cfm_stats;

/* ------------------------------------------------------------------ misc */
int cfm_api_version(void);
const char *cfm_status_string(int status);
const char *cfm_last_error(void);
/* Budget of every device grid-barrier wait, in milliseconds (default 2000). */
int cfm_set_barrier_timeout_ms(double ms);
/* Number of SMs and max co-resident blocks reported for the current device. */
int cfm_device_info(int *num_sms, int *cc_major, int *cc_minor);

/* --------------------------------------------------------------- Jacobi */
typedef struct cfm_jacobi_params {
    int dims;       /* 2 (5-point) or 3 (7-point) */
    int nx, ny, nz; /* grid including fixed columns and halo rows/planes; nz ignored for 2D */
    int precision;  /* cfm_precision */
    int periodic_y; /* 3D only: 1 = rows y=0, ny-1 are periodic halos too (CONFIG problem) */
    int impl;       /* cfm_jacobi_impl */
} cfm_jacobi_params;

typedef struct cfm_jacobi cfm_jacobi;

/* Fill a caller-owned host grid (nx*ny*nz elements of the params' precision)
 * with the initial state of `problem`.  Host-side; needs no GPU.
 * Replaces initialize_boundaries (Stencil/jacobi2D/src/common.cu:15-26,
 * Stencil/jacobi3D/src/common.cu:15-29) plus the zero memsets. */
int cfm_jacobi_problem_host(const cfm_jacobi_params *p, int problem, void *host_grid);

/* Allocate the two device grids of the ping-pong pair and the barrier state. */
int cfm_jacobi_create(const cfm_jacobi_params *p, cfm_jacobi **out);
void cfm_jacobi_destroy(cfm_jacobi *h);
int cfm_jacobi_set_stream(cfm_jacobi *h, void *cuda_stream);
/* x boundary of the 2D sweep. */
typedef enum cfm_boundary {
    /* x = 0 and x = nx-1 are fixed columns, rows 1..ny-2 x 1..nx-2 updated as
     * 0.25 * (((E + W) + N) + S) (jacobi_kernel_single_gpu,
     * Stencil/jacobi2D/src/common.cu:28-42).  The default. */
    CFM_BOUNDARY_DIRICHLET = 0,
    /* every column of rows 1..ny-2 updated, east / west clamped to the cell
     * itself at the x edges, 0.25 * (((N + S) + E) + W): the reference's PERKS
     * comparator jacobi_kernel_single_gpu_mirror (Stencil/jacobi2D/src/
     * common.cu:44-66), which its PERKS run is checked against
     * (Stencil/jacobi2D/src/PERKS/multi-stream-perks.cu:225-226).  Same
     * periodic halo rows.  Every implementation supports it. */
    CFM_BOUNDARY_MIRROR = 1
} cfm_boundary;
/* Select the 2D x boundary for later runs (3D: only CFM_BOUNDARY_DIRICHLET).
 * Replaces the kernel argument of the reference's single_gpu()
 * (Stencil/jacobi2D/src/common.cu:154-156). */
int cfm_jacobi_set_boundary(cfm_jacobi *h, int boundary);
/* Order of the sweeps of the 3D TMA pipeline (persistent and resident
 * implementations): on -- a work unit of sweep t starts once the units
 * around it (distance one, periodic wrap included) have finished sweep
 * t - 1, so no grid-wide barrier; off (default) -- a grid barrier after
 * every sweep, the reference's cg::sync(grid) order
 * (Stencil/jacobi3D/src/single-stream/multi-threaded-two-block-comm.cu:122).
 * Both give the same grid bit for bit; at 512^3 FP64 the barrier order
 * measured 3% faster. */
int cfm_jacobi_set_dataflow(cfm_jacobi *h, int on);
/* Device-side equivalent of cfm_jacobi_problem_host into the handle's grid. */
int cfm_jacobi_load_problem(cfm_jacobi *h, int problem);
/* Copy a caller-owned host grid in / the current grid out (blocking). */
int cfm_jacobi_upload(cfm_jacobi *h, const void *host_grid);
int cfm_jacobi_download(cfm_jacobi *h, void *host_grid);
/* Run `niter` sweeps on the device-resident grid; stats optional.
 * The result equals the reference single_gpu() run for niter sweeps on the
 * same initial grid (Stencil/jacobi3D/src/common.cu:110-239). */
int cfm_jacobi_run(cfm_jacobi *h, int niter, cfm_stats *st);
/* End-to-end call: upload host_in, run niter sweeps, download into host_out.
 * stats->seconds covers both copies and the sweeps. */
int cfm_jacobi_run_host(cfm_jacobi *h, int niter, const void *host_in, void *host_out,
                        cfm_stats *st);
/* Device pointer of the current grid (valid until the next run/destroy). */
void *cfm_jacobi_device_grid(cfm_jacobi *h);
/* Blocks and threads the persistent kernels launch with on this device. */
int cfm_jacobi_launch_shape(cfm_jacobi *h, int *blocks, int *threads);
/* Autotuner for the 3D TMA pipeline: times every compiled pipeline shape for
 * `sweeps` sweeps on a saved copy of the current grid, keeps the fastest for
 * this handle and restores the grid.  best_variant is -1 when the handle does
 * not use the TMA pipeline (2D, host loops, nx * esize not a multiple of 16).
 * Tuning knob (no reference counterpart; the reference hard-codes its launch
 * geometry, Stencil/jacobi3D/src/multi-stream/multi-gpu-peer-tiling.cu:214-220). */
int cfm_jacobi_autotune(cfm_jacobi *h, int sweeps, int *best_variant, double *best_glups);
/* Shape of compiled pipeline variant `index` (CFM_BAD_ARG past the last). */
int cfm_jacobi_variant_info(int index, int *consumer_warps, int *rows_per_warp, int *stages);
/* Sweeps per pass over the grid of pipeline shape `index`: 1, or 2 for the
 * temporally blocked shapes (an odd sweep count ends with one one-sweep
 * launch); a negative status for an unknown index. */
int cfm_jacobi_variant_sweeps(int index);
/* z-chunk (planes per work unit) the 3D persistent kernel of this handle
 * uses (after cfm_jacobi_autotune: the chosen one). */
int cfm_jacobi_zchunk(cfm_jacobi *h);

/* ------------------------------------------------------------------- CG */
typedef enum cfm_cg_impl {
    /* "Single GPU Discrete Standard": kernel per operation, host reads the
     * dots every iteration (CG/src/common.cu:399-538) */
    CFM_CG_DISCRETE = 0,
    /* "Single Stream Standard": whole CG in one persistent kernel
     * (CG/src/single-stream/standard.cu:158-299) */
    CFM_CG_PERSISTENT = 1,
    /* "Single Stream Pipelined" (CG/src/single-stream/pipelined.cu:176-330):
     * one persistent kernel, one fused pass and one grid barrier per iteration */
    CFM_CG_PERSISTENT_PIPELINED = 2,
    /* FP32 persistent CG with FP64 reliable updates (the correction is added
     * to x and the residual replaced by b - A x in FP64, keeping the search
     * direction), one persistent kernel (no reference counterpart; needs
     * tol > 0) */
    CFM_CG_MIXED = 3
} cfm_cg_impl;

typedef struct cfm_csr cfm_csr;

/* Upload a CSR matrix from caller-owned host arrays.  The index base (0 or 1)
 * is taken from rowptr[0], as the reference's main does (CG/src/main.cu:180-187). */
int cfm_csr_create(int n, long long nnz, const int *rowptr, const int *col, const double *val,
                   cfm_csr **out);
void cfm_csr_destroy(cfm_csr *A);
/* MatrixMarket coordinate file -> CSR on the host, with the behaviour of the
 * reference's loadMMSparseMatrix (CG/src/mmio_wrapper.cpp:170-378): real or
 * integer field; general, symmetric, hermitian or skew-symmetric (expanded
 * to the full pattern); entries sorted by (row, column); the index base of
 * the file (1 when an index equals the dimension, 0 when one is 0) kept in
 * rowptr[0], as cfm_csr_create expects.  Call first with rowptr = NULL for
 * *m, *n and *nnz, then with rowptr (m + 1), col and val (nnz) allocated.
 * Dense (array), pattern and complex files are CFM_UNSUPPORTED. */
int cfm_mm_read(const char *path, int *m, int *n, long long *nnz, int *rowptr, int *col, double *val);
/* y = A x with host vectors (FP64, deterministic row order). */
int cfm_csr_spmv_host(const cfm_csr *A, const double *x, double *y);

/* Matrix-free variable-coefficient operator -div(k grad u) on a 2D (5-point)
 * or 3D (7-point) grid of unit cells, u = 0 on the boundary; face
 * coefficients are harmonic means 2 k_i k_j / (k_i + k_j), boundary faces
 * 2 k_i (cfm_varcoef_coeffs).  Rows are cells, x fastest.  No reference
 * counterpart (the reference's CG takes CSR only, CG/src/main.cu:118-135). */
typedef struct cfm_stencil cfm_stencil;
int cfm_stencil_create(int dims, int nx, int ny, int nz, const double *k_host, cfm_stencil **out);
void cfm_stencil_destroy(cfm_stencil *S);
/* y = A x with host vectors. */
int cfm_stencil_apply_host(const cfm_stencil *S, const double *x, double *y);

typedef struct cfm_cg_params {
    int impl;          /* cfm_cg_impl */
    int maxiter;       /* iteration cap (CFM_CG_MIXED: FP32 iterations);
                          with tol <= 0 exactly maxiter iterations run */
    double tol;        /* relative residual target ||r||/||b||; <= 0 = fixed count (reference -niter) */
    int inner_maxiter; /* CFM_CG_MIXED: most FP32 iterations between two FP64 updates (0 = no cap) */
    double inner_tol;  /* CFM_CG_MIXED: an FP64 update when |r| falls below inner_tol times its
                          largest norm since the last one (0 = default 0.1) */
} cfm_cg_params;

typedef struct cfm_cg cfm_cg;

int cfm_cg_create(const cfm_csr *A, const cfm_cg_params *p, cfm_cg **out);
/* CG handle over a matrix-free stencil operator (same solvers as CSR). */
int cfm_cg_create_stencil(const cfm_stencil *S, const cfm_cg_params *p, cfm_cg **out);
void cfm_cg_destroy(cfm_cg *h);
int cfm_cg_set_stream(cfm_cg *h, void *cuda_stream);
/* Solve A x = b from x0 = 0 with host vectors; b == NULL means b = ones, the
 * reference's right-hand side (CG/src/common.cu:133-140). */
int cfm_cg_solve(cfm_cg *h, const double *b_host, double *x_host, cfm_stats *st);
/* Same with device vectors (length n, FP64). */
int cfm_cg_solve_device(cfm_cg *h, const double *b_dev, double *x_dev, cfm_stats *st);

/* Largest system cfm_cg_solve_noalloc accepts (rows). */
#define CFM_CG_NOALLOC_MAX_N 262144

/* Persistent CG (the CFM_CG_PERSISTENT kernel and arithmetic, so the same x
 * and iteration count) for callers that cannot allocate device memory: code
 * that runs inside another framework's memory pool or allocator, in a
 * process whose device memory is reserved up front, or at a point where an
 * allocation would synchronise the device.  It calls no cudaMalloc,
 * cudaFree, stream or event creation.  Its working vectors (r, p, s, t), dot
 * partials, result word and grid-barrier state live in one fixed device
 * array inside the library, about 8.0 MiB, that every GPU which loads the
 * library holds until the process exits.
 *  - Inputs and outputs are the caller's device memory: a 0-based CSR
 *    matrix (rowptr n+1, col nnz, val nnz) with n <= CFM_CG_NOALLOC_MAX_N
 *    (larger n: CFM_BAD_ARG), b (NULL = ones) and x (length n, written).
 *    b and x must be different arrays (CFM_BAD_ARG otherwise).
 *  - Work goes on `cuda_stream` (NULL = the legacy default stream); the
 *    call waits for that stream and reads the result back before it
 *    returns.  stats->seconds is host time.
 *  - Set-up: the first call on a device looks up the array's device address
 *    with that device current; make that first call before any stream
 *    capture.  With lazy module loading (the CUDA default) this first call is
 *    also what loads the array onto the device, so it may allocate device
 *    memory itself: make it (a 1-row system is enough) before the caller
 *    reserves or hands out its memory.  Out of memory there is
 *    CFM_OUT_OF_MEMORY.  The address is kept for the process: calls after a
 *    cudaDeviceReset of that device are not supported.
 *  - All calls share the one array and the call resets what must start at
 *    zero, so calls whose kernels overlap on the GPU (other threads, other
 *    streams) race; serialise them.
 * No counterpart in the reference: its CG versions allocate their vectors
 * themselves with cudaMalloc. */
int cfm_cg_solve_noalloc(int n, long long nnz, const int *rowptr_dev, const int *col_dev,
                         const double *val_dev, const double *b_dev, double *x_dev, int maxiter,
                         double tol, void *cuda_stream, cfm_stats *st);

/* ------------------------------------------------------------ generators */
/* Number of nonzeros of the 7-point Dirichlet Poisson matrix on gx*gy*gz cells. */
long long cfm_poisson3d_nnz(int gx, int gy, int gz);
/* 7-point Poisson matrix (diagonal 6, off-diagonals -1, Dirichlet boundary
 * eliminated), 0-based CSR with sorted columns, into caller arrays of size
 * n+1, nnz, nnz. */
int cfm_poisson3d_csr(int gx, int gy, int gz, int *rowptr, int *col, double *val);
/* The reference's random tridiagonal test matrix (CG/src/common.cu:46-76),
 * drawn from libc rand() in its default state; nnz = 3n-2. */
int cfm_tridiag_csr(int n, int *rowptr, int *col, double *val);
/* n doubles uniform in [lo, hi) from a Philox-4x32-10 stream keyed by seed. */
int cfm_uniform(unsigned long long seed, long long n, double lo, double hi, double *out);

/* n doubles ~ N(0, 1): Box-Muller on Philox-4x32-10 words, counter
 * (i / 2, stream), key seed. */
int cfm_normal(unsigned long long seed, unsigned int stream, long long n, double *out);
/* Gaussian random field on an nx*ny(*nz) grid: Philox white noise convolved
 * (periodic wrap) with a separable Gaussian kernel, unit variance before the
 * sigma scale, covariance exp(-r^2 / (2 corr_len^2)). */
int cfm_grf(int dims, int nx, int ny, int nz, unsigned long long seed, double sigma,
            double corr_len, double *g);
/* Variable-coefficient diffusion problem: k = exp(grf(sigma 1, corr_len 16)),
 * f ~ N(0, 1) per cell (stream 1). */
int cfm_varcoef_problem(int dims, int nx, int ny, int nz, unsigned long long seed, double *k,
                        double *f);
/* Face coefficients of cfm_stencil from k: w_e/w_n/w_t = faces to x+1/y+1/z+1
 * (0 on the last column/row/plane), diag = sum of the cell's face weights
 * (boundary faces 2 k_i) in the order x-, x+, y-, y+, z-, z+.  w_t unused in 2D. */
int cfm_varcoef_coeffs(int dims, int nx, int ny, int nz, const double *k, double *w_e,
                       double *w_n, double *w_t, double *diag);

/* One Philox-4x32-10 block (counter, key) -> 4 words; the generator behind
 * cfm_uniform, exported for its known-answer test. */
int cfm_philox4x32_10(const unsigned int ctr[4], const unsigned int key[2], unsigned int out[4]);

/* ------------------------------------------- tensor-core convolutions */
/* The 3x3 convolutions of the learned preconditioner on the tcgen05 tensor
 * cores (BF16 operands, FP32 accumulation in TMEM), run once on host buffers.
 * No reference counterpart (the reference has no tensor-core code); exposed
 * for parity tests of the kernels.  BF16 values are passed as their 16-bit
 * patterns.  Layouts: x [B][H][W][Cin], w [9][Cout][Cin] (tap = 3 dy + dx,
 * padding 1), out [B][H][W][Cout]; Cin a multiple of 32 up to 256, Cout in
 * {32, 64, 128, 256}, W a power of two up to 128 or a multiple of 128.
 * out = relu?(conv(x, w) + bias), rounded to BF16. */
int cfm_tc_conv3x3(int B, int H, int W, int Cin, int Cout, const unsigned short *x,
                   const unsigned short *w, const float *bias, int relu, unsigned short *out);
/* Weight gradient dw[tap][co][ci] = sum over pixels p of
 * dz[p][co] * x[p + (dy - 1, dx - 1)][ci] (zero outside), FP32; W a
 * multiple of 32. */
int cfm_tc_conv3x3_wgrad(int B, int H, int W, int Cin, int Cout, const unsigned short *x,
                         const unsigned short *dz, float *dw);

/* ------------------------------------------------ learned preconditioner */
/* The U-Net of the learned preconditioner (no reference counterpart):
 * 4 levels (H, H/2, H/4, H/8) with 32/64/128/256 channels, 3x3 convolutions
 * with bias and ReLU, 2x2 mean pooling, nearest upsampling with additive
 * skips; input [B][H][W][2] FP32 (normalised residual, log k), output
 * [B][H][W] FP32.  Wide convolutions on the tcgen05 tensor cores (BF16,
 * FP32 accumulate).  Parameters: one flat FP32 vector, per layer
 * (cin 2->32, e1 32->64, e2 64->128, e3 128->256, d3 256->128, d2 128->64,
 * d1 64->32, d0 32->32, cout 32->1) weight [9][Cout][Cin] then bias [Cout].
 * H a multiple of 8, W a multiple of 256. */
typedef struct cfm_unet cfm_unet;
long long cfm_unet_num_params(void);
int cfm_unet_create(int H, int W, int max_batch, unsigned long long seed, cfm_unet **out);
void cfm_unet_destroy(cfm_unet *net);
int cfm_unet_get_params(cfm_unet *net, float *theta);
int cfm_unet_set_params(cfm_unet *net, const float *theta);
/* Records what a network restored with cfm_unet_set_params was trained for
 * (smoothing sweeps 0..8, coarsening 1 or 2), as cfm_unet_train_varcoef
 * does, so that cfm_fpcg_create accepts it. */
int cfm_unet_set_training_info(cfm_unet *net, int smooth, int coarsen);
/* One forward pass on host buffers. */
int cfm_unet_forward_host(cfm_unet *net, int B, const float *in, float *out);
/* Forward, then the gradient of sum(out * dout) with respect to the
 * parameters into grad (cfm_unet_num_params floats). */
int cfm_unet_gradient_host(cfm_unet *net, int B, const float *in, const float *dout, float *grad);
/* Device time of one forward pass of batch B on device-resident buffers:
 * one pass captured in a CUDA graph (as a solver's graph runs it), replayed
 * `iters` times back to back after a warm-up; CUDA events. */
int cfm_unet_time_forward(cfm_unet *net, int B, int iters, double *ms_per_forward);
/* Which forward pass the network runs (no counterpart in the reference,
 * whose solver has no learned preconditioner):
 *   CFM_UNET_FORWARD_LAYERS      one kernel per layer (19 launches, PDL);
 *   CFM_UNET_FORWARD_PERSISTENT  one persistent cooperative kernel that walks
 *                                the layers behind bounded grid barriers;
 *   CFM_UNET_FORWARD_AUTO        (default) the per-layer kernels, which
 *                                measured faster at every size tried.
 * Both give bit-identical outputs.  The persistent pass fails with
 * CFM_UNSUPPORTED when a layer's staging does not fit its shared ring.  A
 * solver that captured the forward in its graph keeps the pass it captured
 * until it builds the graph again. */
enum {
    CFM_UNET_FORWARD_AUTO = 0,
    CFM_UNET_FORWARD_LAYERS = 1,
    CFM_UNET_FORWARD_PERSISTENT = 2
};
int cfm_unet_set_forward_mode(cfm_unet *net, int mode);
/* Device time of one training step at batch B (forward, the backward pass
 * of sum(out * dout) with its weight gradients, one Adam step at lr 1e-4)
 * on fixed synthetic inputs, averaged over `iters` steps after one warm-up
 * step.  It trains the network on those inputs: time a scratch network. */
int cfm_unet_time_train_step(cfm_unet *net, int B, int iters, double *ms_per_step);
/* BF16 patterns of one activation of the last forward pass (testing): index
 * 0..13 = h0 p1 h1 p2 h2 p3 h3 g3 u2 g2 u1 g1 u0 g0, NHWC at its level. */
int cfm_unet_activation_host(cfm_unet *net, int which, int B, unsigned short *out);

/* Training of the network for the 2D variable-coefficient problem on the
 * (coarsen H) x (coarsen W) grid of an H x W network (coarsen 1 or 2):
 * nsys systems from fresh seeds seed0, seed0+1, ... (k = exp(GRF),
 * f ~ N(0,1), cfm_varcoef_problem) are solved by plain persistent FP64 CG to
 * 1e-10; from a second run, `snaps` iterates x_j spread over the solve plus
 * x_0 = 0 give (snaps + 1) * nsys residual/error pairs (r_j = f - A x_j,
 * e_j = x* - x_j); then `epochs` shuffled passes of Adam (lr, batch <=
 * the net's max_batch) on the per-sample energy-norm loss
 * 1 - <z, r_j>^2 / (<z, A z> <e_j, r_j>), z = net(r_j): one minus the share
 * of ||e_j||_A^2 that one CG step along z removes.
 * Mean loss of the first and last epoch and the seconds spent on data and on
 * training are returned (each pointer optional).  smooth > 0: every pair is
 * first passed through `smooth` damped Jacobi sweeps z on A z = r_j, giving
 * (r_j - A z, e_j - z), the pair the network sees inside the preconditioner.
 * With coarsen = 2 the network sees the residual restricted to its grid
 * (2 x 2 means of r_j / rms(r_j), block-mean log k) and z = P net(.) is its
 * piecewise-constant prolongation; the loss is taken on the systems' grid. */
int cfm_unet_train_varcoef(cfm_unet *net, int nsys, int snaps, unsigned long long seed0, int epochs,
                           int batch, float lr, int smooth, int coarsen, double *loss_first,
                           double *loss_last, double *data_seconds, double *train_seconds);
/* Checkpoint selection for cfm_unet_train_varcoef: with every > 0, one
 * held-out variable-coefficient system (cfm_varcoef_problem with `seed`, the
 * training systems' size) is solved to 1e-8 by FPCG (the defaults with a
 * network) with the network as it trains, after every `every` epochs and
 * after the last; training ends with the parameters of the solve that took
 * the fewest iterations (ties: the earlier epoch).  every = 0 (default)
 * keeps the last epoch's.  Training is deterministic: every gradient, loss
 * and data sum is added in a fixed order, so the same seeds give the same
 * parameters and the same kept epoch on every run. */
int cfm_unet_set_validation(cfm_unet *net, unsigned long long seed, int every);
/* The kept checkpoint of the last training: epochs trained (-1: no
 * validation) and its FPCG time on the validation system (ms). */
int cfm_unet_validation(const cfm_unet *net, int *best_epoch, double *best_ms);

/* Flexible PCG (truncated FCG(m): each direction A-orthogonalised against
 * the last m, alpha = <p, r> / <p, A p>) on a 2D stencil operator with the
 * preconditioner z = J(z0 + c y): z0 = J(0), r1 = r - A z0,
 * y = net(r1 / |r1|_rms, log k), c = <y, r1> / <y, A y> (the optimal step
 * along y), J = `smooth` damped Jacobi sweeps (omega 0.8, smooth <= 8) on A z = r;
 * k_host the cell coefficients the stencil was built from; smooth must
 * equal the value the network was trained with.  FP64 vectors and dots; one
 * CUDA graph whose conditional while-node runs the iterations on the device.
 * If the loop stalls or reaches maxiter, plain persistent FP64 CG finishes
 * from the current iterate; stats->refinements = 1 then.  stats->iterations
 * = FPCG iterations + fallback iterations; stats->lups = FPCG iterations.
 * The stencil's grid must be the network's times the factor it was trained
 * with (cfm_unet_train_varcoef coarsen); with factor 2 the network sees
 * R(r1) (2 x 2 means) and y above is P net(.), its piecewise-constant
 * prolongation (a learned coarse-grid correction). */
typedef struct cfm_fpcg cfm_fpcg;
int cfm_fpcg_create(const cfm_stencil *S, const double *k_host, cfm_unet *net, int smooth,
                    int maxiter, double tol, cfm_fpcg **out);
void cfm_fpcg_destroy(cfm_fpcg *h);
/* Truncation m in [1, 8] of the orthogonalisation (default 8 with a
 * network, 1 without); m = 1 is the Polak-Ribiere-like one-term recurrence. */
int cfm_fpcg_set_truncation(cfm_fpcg *h, int m);
/* Apply the network in one of every `every` iterations (1..8; default 2
 * with a network); the others use the smoothing alone (c = 0). */
int cfm_fpcg_set_network_period(cfm_fpcg *h, int every);
/* Precision of the Krylov iteration.  CFM_FP64 (default): FP64 vectors,
 * recurrences and dots.  CFM_FP32: mixed precision with FP64 reliable
 * updates -- the residual, directions, A p and the correction are FP32 and
 * A p uses the FP32 coefficients; dots are FP64 sums of the exact FP32
 * products and alpha, beta are FP64 (applied rounded to FP32); the iterate is
 * x = x64 + d32.  When |r32| reaches tol |b| or falls below delta times its
 * largest value since the last update, x64 += d32 in FP64, d32 = 0 and r32 is
 * replaced by fl32(b - A x64) from the FP64 true residual, which alone
 * decides convergence; the directions are kept (the reliable-update scheme
 * of CFM_CG_MIXED).  The preconditioner is unchanged (FP32 smoothing, BF16
 * network); plain FP64 CG stays the fallback.  No counterpart in the
 * reference (its CG is FP64 only). */
int cfm_fpcg_set_precision(cfm_fpcg *h, int precision, double delta);
/* FP64 reliable updates of the last solve (0 in FP64 mode). */
int cfm_fpcg_reliable_updates(const cfm_fpcg *h);
/* How a single system's iterations run on the device.  on = 0 (default):
 * one kernel per phase, chained by programmatic dependent launch inside the
 * solver's CUDA graph.  on = 1: the solver kernels between two network
 * applications run as one persistent cooperative launch that walks the
 * phases behind bounded grid barriers (the persistent-kernel idea of the
 * reference's CPU-free CG, CG/src/single-stream/standard.cu:158-299,
 * applied to FPCG).  Both compute the same values bit for bit; on B200 the
 * per-phase kernels measured faster (512^2: 38 against 48 ms for
 * Jacobi-smoothed FPCG).  Batches always use the per-phase kernels. */
int cfm_fpcg_set_device_loop(cfm_fpcg *h, int on);
/* A batch of independent 2D variable-coefficient systems solved together
 * by the same device loop: member m has cells nx[m] x ny[m] and
 * coefficients k_host[m] (built as cfm_varcoef_coeffs does).  Every member
 * is embedded at the origin of one frame -- the network's grid times its
 * factor, or with net == NULL the largest member -- whose padding is a
 * decoupled identity block with zero right-hand side, so it stays zero; the
 * network runs on all members' frames at once (in chunks of its largest
 * batch) and its correction is kept inside each member.  Each member has its
 * own scalars, convergence test and iteration count; converged members stop
 * while the others go on (one conditional graph).  Precision, truncation and
 * network period are set as for one system.  No counterpart in the
 * reference. */
int cfm_fpcg_create_batch(int nmem, const int *nx, const int *ny, const double *const *k_host,
                          cfm_unet *net, int smooth, int maxiter, double tol, cfm_fpcg **out);
/* Solves member m for b_host[m] into x_host[m] (row-major nx[m] x ny[m]);
 * per-member iterations, status (CFM_OK when the FP64 true relative residual
 * reached tol) and true relative residual (each optional).  Returns CFM_OK or
 * CFM_NOT_CONVERGED if any member did not converge.  stats: the whole
 * batch (seconds, the largest iteration count, launches). */
int cfm_fpcg_solve_batch(cfm_fpcg *h, const double *const *b_host, double *const *x_host,
                         long long *iters, int *status, double *relres, cfm_stats *st);
int cfm_fpcg_solve(cfm_fpcg *h, const double *b_host, double *x_host, cfm_stats *st);
/* Recursive residual norms |r_k| of the last solve, one per iteration from
 * k = 0 (at most max_n; *n_out = the count).  net == NULL in
 * cfm_fpcg_create gives the identity preconditioner (plain CG in the same
 * device loop). */
int cfm_fpcg_history(cfm_fpcg *h, double *out, long long max_n, long long *n_out);

/* ------------------------------------------------------- batched solves */
/* Many independent variable-coefficient systems (2D 5-point / 3D 7-point,
 * uneven sizes) solved in ONE persistent cooperative launch captured in a
 * CUDA graph (no reference counterpart).  The resident blocks form teams
 * per size class; each team takes systems from its class queue (largest
 * first) and solves them with PCG (FP64, or FP32 inside FP64 refinement:
 * cfm_batch_set_precision; damped-Jacobi polynomial preconditioner) behind
 * team-local bounded barriers.  System i: dims[i],
 * nx/ny/nz[i] (nz ignored in 2D), cell coefficients k_host[i] and right-hand
 * side b_host[i] (x0 = 0). */
typedef struct cfm_batch cfm_batch;
int cfm_batch_create(int nsys, const int *dims, const int *nx, const int *ny, const int *nz,
                     const double *const *k_host, const double *const *b_host, cfm_batch **out);
void cfm_batch_destroy(cfm_batch *h);
/* Size classes: class c takes the systems with n >= thresholds[c] not taken
 * by an earlier class (thresholds descending, the last 0), on teams of
 * team_sizes[c] blocks; blocks are shared in proportion to class work. */
int cfm_batch_set_plan(cfm_batch *h, int ncls, const long long *thresholds, const int *team_sizes);
/* smooth damped Jacobi sweeps in the preconditioner (0 = diagonal scaling),
 * iteration cap, relative tolerance (defaults 4, 20000, 1e-8). */
int cfm_batch_set_solver(cfm_batch *h, int smooth, int maxiter, double tol);
/* CFM_FP64 (default): PCG in FP64.  CFM_FP32: mixed-precision PCG with
 * reliable updates, per system in the same persistent launch: the iteration
 * runs in FP32 (FP32 copies of the coefficients, FP32 preconditioner and
 * vectors; dots as FP64 sums of exact FP32 products; alpha, beta in FP64)
 * and gathers its steps in an FP32 correction; when the recursive residual
 * falls below the tolerance, below inner_tol (0: 0.1) times its largest
 * norm since the last update, or after inner_maxiter steps (0: no cap), the
 * correction is added to x in FP64 and r is replaced by the FP64 true
 * residual b - A x, keeping the search direction.  It stops on the FP64
 * true residual |b - A x| <= tol |b|; stats->refinements = the sum of
 * updates. */
int cfm_batch_set_precision(cfm_batch *h, int precision, int inner_maxiter, double inner_tol);
/* Solve all systems (one graph launch).  Per system (each array optional):
 * iterations, status, FP64 true relative residual; stats->seconds = device
 * time of the launch, stats->iterations = the sum of iterations. */
int cfm_batch_solve(cfm_batch *h, long long *iters, int *status, double *relres, cfm_stats *st);
int cfm_batch_solution(cfm_batch *h, int i, double *x_host);
/* Autotuner: times every built-in plan (class thresholds x team sizes) on
 * the real batch and keeps the fastest. */
int cfm_batch_autotune(cfm_batch *h, double *best_ms);

/* -------------------------------------------------------------- testing */
/* Launch a persistent kernel of `blocks` blocks (0 = device default) that
 * meets `rounds` grid barriers; when drop_block >= 0 that block skips its
 * arrival at the first barrier.  Returns CFM_OK or CFM_BARRIER_TIMEOUT; the
 * device stays usable either way. elapsed_ms (optional) gets the kernel time. */
int cfm_barrier_selftest(int blocks, int rounds, int drop_block, double *elapsed_ms);

#ifdef __cplusplus
}
#endif

#endif /* CFM_H */
