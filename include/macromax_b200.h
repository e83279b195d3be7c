/*
 * macromax_b200 -- C ABI of the B200-native split-Richardson (modified Born) solver.
 *
 * Every entry point takes plain pointers and sizes; device pointers are CUDA device memory of the device that was
 * current when the plan was created, `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 * Functions return MMX_OK (0) on success and a negative code on failure; mmx_last_error() then describes the
 * failure (thread-local, valid until the next call on the same thread).
 *
 * Data layout (C order, complex words interleaved re/im; complex64 = 8 bytes, complex128 = 16 bytes):
 *   field  [batch][ncomp][n0][n1][n2]      ncomp = 1 (scalar) or 3 (vector); the reference's [c, 1, *grid]
 *   chi    [m][n0][n1][n2]                  m = 1 (isotropic) or 9 (3x3, row-major); the reference's [r, r, *grid]
 *   source [batch][ncomp][n0][n1][n2]      the preconditioned source s' = i s / (alpha_i beta)
 * Each call replaces a call site of the reference MacroMax Python package (paths relative to python/macromax).
 */
#ifndef MACROMAX_B200_H
#define MACROMAX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MMX_OK 0
#define MMX_ERR_ARG (-1)
#define MMX_ERR_CUDA (-2)
#define MMX_ERR_UNSUPPORTED (-3)

#define MMX_C64 0  /* complex64 words  */
#define MMX_C128 1 /* complex128 words */

#define MMX_CHI_SCALAR 1 /* isotropic susceptibility, one word per voxel */
#define MMX_CHI_MAT3 9   /* 3x3 susceptibility tensor, nine words per voxel */
#define MMX_CHI_SYM6 6   /* symmetric 3x3 tensor, six words per voxel: xx, xy, xz, yy, yz, zz */

/* status codes of an mmx_rhs_state */
#define MMX_STATUS_OK 0
#define MMX_STATUS_ZERODIV 1 /* update norm 0 after a previous norm of 0: the reference raises ZeroDivisionError */
#define MMX_STATUS_TIMEOUT 2 /* a bounded wait for an asynchronous shared-memory copy gave up (results kept valid) */

/*
 * Per right-hand-side iteration state, one entry per batch member, in DEVICE memory.  Mirrors the private state of
 * Solution (solver.py:161, 474, 997-1047): alpha, previous_update_norm, iteration, residue.  chi and the source are
 * stored once, at alpha0; the iteration applies chi(alpha) = chi0 alpha0_i / alpha_i + i (alpha0 - alpha) / alpha_i
 * and s'(alpha) = s'0 alpha0_i / alpha_i on the fly, which is what __update_operators (solver.py:496-528) does to
 * the stored arrays when the divergence guard raises alpha_i.
 */
typedef struct mmx_rhs_state {
  double alpha_re, alpha_im;   /* current alpha */
  double alpha0_re, alpha0_im; /* alpha at which chi and source were stored */
  double prev_norm;            /* previous_update_norm, +inf after a reset (solver.py:161, 720, 832) */
  double last_norm;            /* ||d|| of the last iteration */
  double field_norm;           /* ||E|| of the current field (times k0^2) */
  double residue;              /* previous_update_norm / ||E|| (solver.py:1026-1042) */
  double rtol;                 /* keep iterating while residue > rtol ... */
  double maxiter;              /* ... and iteration < maxiter (solver.py:81-83) */
  int32_t iteration;           /* iterations since the last reset of the counter */
  int32_t cur;                 /* which of the two field buffers holds the current E */
  int32_t active;              /* 1 while the stop rule asks for more iterations */
  int32_t accepted;            /* 1 if the last update was accepted by the divergence guard */
  int32_t rejections;          /* number of rejected updates (alpha_i raised by 1.5x) */
  int32_t status;              /* MMX_STATUS_* */
  int32_t reserved[2];         /* [0]: used by mmx_magnetic_iterate.  [1]: bit c set = component c of this right-hand
                                  side's source is identically zero, so the prologue may skip reading it; 0 claims
                                  nothing.  Whoever writes the source clears or sets it (mmx_defect's output, for
                                  instance, is a dense source: clear the bits of the states that read it). */
} mmx_rhs_state;

typedef struct mmx_plan mmx_plan;

/* Human-readable description of the last failure on this thread. */
const char* mmx_last_error(void);

/* ABI version of this library. */
int mmx_version(void);

/*
 * Create a plan for fields on a periodic grid of `ndim` (1..3) axes with lengths `shape` (C order), `ncomp` (1|3)
 * components, `batch` right-hand sides and word `precision` (MMX_C64 | MMX_C128) on the current CUDA device.
 * Replaces the grid / dtype / working-array set-up of BackEnd.__init__ (backend/__init__.py:43-67) and
 * backend.load (backend/__init__.py:922-1012).  Axis lengths must factor into 2, 3, 5, 7, 11, 13.
 */
int mmx_plan_create(int ndim, const int64_t* shape, int ncomp, int batch, int precision, mmx_plan** plan);

/* Release a plan and its device memory (twiddles, k tables, work buffers). */
int mmx_plan_destroy(mmx_plan* plan);

/*
 * Set the k-vectors of the k0-scaled grid: for each axis a, shape[a] values k_a[j] (origin at index 0), concatenated
 * over the axes (host memory, FP64).  Replaces BackEnd.k (backend/__init__.py:651-656; utils/ft/grid.py:426-439).
 */
int mmx_plan_set_kvectors(mmx_plan* plan, const double* k);

/*
 * N-D discrete Fourier transform over the grid axes of `nbatch` contiguous fields of the plan's shape and precision
 * (in == out allowed).  inverse = 0: forward, unscaled; inverse = 1: inverse scaled by 1/N, so that
 * ift(ft(x)) == x.  Replaces BackEnd.ft / BackEnd.ift (backend/__init__.py:234-257; numpy backend
 * backend/numpy.py:112-133; torch backend backend/torch.py:183-205).
 */
int mmx_fftn(mmx_plan* plan, const void* in, void* out, int64_t nbatch, int inverse, void* stream);

/*
 * ||x||_2 of `nwords` complex words of the given precision, accumulated in FP64, written to out_dev[0] (device).
 * Uses the plan's scratch.  Replaces BackEnd.norm (backend/__init__.py:872-874; backend/torch.py:316-317).
 */
int mmx_norm(mmx_plan* plan, const void* x, int64_t nwords, int precision, double* out_dev, void* stream);

/*
 * Run `niter` iterations of Solution.__iter__ (solver.py:1049-1098) for every active right-hand side:
 *   d = chi [G (chi E + s') - E],  accept E += d if ||d|| < previous_update_norm, else alpha_i *= 1.5,
 * with G = IFFT g(k) FFT, g = -i alpha_i / (|k|^2 - alpha) for scalar fields and the transverse/longitudinal split
 * g (1 - P_L) + (i alpha_i / alpha) P_L for vector fields (solver.py:564-584; backend/__init__.py:606-649).
 * The current field of RHS b is buffer state[b].cur of (E0, E1); the update is written to the other buffer and the
 * two swap roles on acceptance.  A right-hand side whose state is inactive is skipped (convergence mask).
 * chi: chi_kind MMX_CHI_SCALAR, MMX_CHI_MAT3 or MMX_CHI_SYM6 (a symmetric tensor stored as its six distinct
 * entries), shared by all right-hand sides.  All launches are asynchronous on
 * `stream`; no host synchronisation happens inside.
 */
int mmx_iterate(mmx_plan* plan, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                mmx_rhs_state* state, int niter, void* stream);

/*
 * mmx_iterate for `niter` iterations as one CUDA graph launch: the pass kernels are captured once per (plan,
 * buffers, niter) and replayed, which removes the per-kernel launch gaps that dominate small grids.  Same
 * semantics as mmx_iterate.  The captured graph is released with the plan.
 */
int mmx_iterate_graph(mmx_plan* plan, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                      mmx_rhs_state* state, int niter, void* stream);

/* Capture (and cache) the graph that mmx_iterate_graph would launch, without launching it; the graph is uploaded to
 * the device (on the legacy default stream, synchronously), so that its first launch pays no upload either.  Where
 * mmx_iterate_graph_continue would start its chunk with the middle passes now, that graph is captured too. */
int mmx_iterate_graph_prepare(mmx_plan* plan, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                              mmx_rhs_state* state, int niter);

/*
 * mmx_iterate_graph for the next chunk of the same solve.  The caller guarantees that nothing has written the
 * fields, chi, the sources or the states since the previous iteration call on this plan with the same buffers (as
 * between the chunks of Solution.solve, solver.py:1049-1098, which only read the state).  When that call ran the
 * fused-epilogue schedule (MMX_VARIANT_FUSED_EPILOGUE), its last pass left this chunk's first pass -- chi E + s'
 * of the current field, transformed along the contiguous axis -- in the plan's work buffer, so the chunk starts
 * with the middle passes instead of recomputing it; the iterates are those of one longer mmx_iterate_graph call.
 * Otherwise (another plan call came between, the variant changed, other buffers, the plain schedule) it is
 * mmx_iterate_graph.  No counterpart in the reference, whose solve runs every iteration from the field.
 */
int mmx_iterate_graph_continue(mmx_plan* plan, void* E0, void* E1, const void* chi, int chi_kind, const void* src,
                               mmx_rhs_state* state, int niter, void* stream);

/*
 * `niter` iterations of n independent problems (plans of possibly different grid shapes, e.g. an uneven batch of
 * 128^2, 256^2 and 384^2 grids) packed into ONE captured CUDA graph whose branches run concurrently.  Arrays of
 * length n give each plan's buffers as in mmx_iterate.  The reference solves such problems one after another.
 */
int mmx_iterate_multi(int n, mmx_plan* const* plans, void* const* E0, void* const* E1, const void* const* chi,
                      const int* chi_kind, const void* const* src, mmx_rhs_state* const* state, int niter,
                      void* stream);

/*
 * Mixed-precision defect of the FP64 outer loop, for a complex128 plan:
 *   s_out = [s'(alpha) + chi(alpha) x - G(alpha)^{-1} x] alpha_i / alpha0_i      (complex128 in, complex64 out)
 * i.e. the source, normalised to alpha0 like every stored source, for which the plain iteration's fixed point is
 * the correction to x.  Uses state[b].alpha and alpha0 as mmx_iterate does.  No reference counterpart: the
 * reference iterates in one precision.
 */
int mmx_defect(mmx_plan* plan, const void* x, const void* chi, int chi_kind, const void* src,
               const mmx_rhs_state* state, void* s_out, void* stream);

/* x (complex128) += delta (complex64), `nwords` words.  Solution accumulation of the FP64 outer loop. */
int mmx_accumulate(void* x, const void* delta, int64_t nwords, void* stream);

/*
 * Adjoint-state gradient of a real loss with respect to the permittivity, per voxel:
 *   grad[b][v] = scale * conj( sum_c nu[b][c][v] * E[b][c][v] )   (isotropic, ncomp components)
 * where nu solves the adjoint problem with source conj(dL/dE) (torch convention).  No reference counterpart.
 */
int mmx_adjoint_grad(const void* E, const void* nu, void* grad, int64_t batch, int ncomp, int64_t nvox,
                     int precision, double scale, void* stream);

/*
 * Pointwise matrix product out = A B of matrix fields (BackEnd.mul, backend/__init__.py:415-444;
 * backend/torch.py:220-249): A [ra][ca][N], B [ca][cb][N] (B's voxel stride 0 if b_broadcast), out [ra][cb][N].
 */
int mmx_pointwise_mul(const void* A, int ra, int ca, const void* B, int cb, int b_broadcast, void* out,
                      int64_t nvox, int precision, void* stream);

/* Kernel variants of a plan (bit flags), chosen by the autotuner (macromax_b200/autotune.py). */
#define MMX_VARIANT_GENERIC 1u        /* runtime-length shared-memory kernels only */
#define MMX_VARIANT_SHARED_STAGED 2u  /* compile-time kernels without the register-staged passes */
#define MMX_VARIANT_PERSISTENT 4u     /* persistent double-buffered prologue/epilogue passes */
#define MMX_VARIANT_PLANE 8u          /* 3D, 128 x 128 planes, isotropic chi: the two inner axes in one pass */
#define MMX_VARIANT_FUSED_EPILOGUE 16u /* epilogue fused with the next prologue (speculative); isotropic chi, and a 3x3 chi on 192-sample rows */
#define MMX_VARIANT_TMA 32u            /* strided 128-sample passes staged by bulk tensor (TMA) copies */

/* Select the kernel variant of a plan (rebuilds its pass list, drops its captured graphs).  No reference
 * counterpart: the reference has one implementation per backend. */
int mmx_plan_set_variant(mmx_plan* plan, unsigned flags);
unsigned mmx_plan_get_variant(const mmx_plan* plan);

/*
 * Set-up reductions over a 3x3 complex128 matrix field M [9][nvox] (row-major entries), FP64, written to
 * out_dev[0..1] (device):
 *   mode 0: out_dev[1] = max over voxels of the largest eigenvalue of (ab I - M)^H (ab I - M), the alpha objective
 *           sqrt(largest_eigenvalue(...)) of solver.py:392-401 (via mat3_eigh, backend/__init__.py:670-850);
 *   mode 1: out_dev[0], out_dev[1] = min and max over voxels of the eigenvalues of -0.5i (M - M^H), the gain/loss
 *           test of solver.py:322-336.
 * Eigenvalues in closed form (trigonometric solution of the characteristic cubic; like the reference's own cubic
 * roots, accurate to ~1e-8 relative where the largest eigenvalue is (nearly) double).  Uses the plan's scratch.
 */
int mmx_mat3_extremes(mmx_plan* plan, const void* M, int64_t nvox, int mode, double ab, double* out_dev,
                      void* stream);

/*
 * Magnetic and bi-(an)isotropic media (solver.py:531-552): the susceptibility operator
 * chi(x) = chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x), D = the spectral curl (backend/__init__.py:472-509), is
 * composed on the host from mmx_fftn and these kernels.  Fields are [3][N] in the plan's precision; k are the plan's
 * k-vectors (mmx_plan_set_kvectors, k0-scaled grid).
 *   mmx_curl_ft:  out = i k x F for a spectrum F (not in place).            Replaces BackEnd.curl_ft (:483-509).
 *   mmx_green_ft: F <- g (F - P_L F) + (i alpha_i / alpha) P_L F in place,   Replaces g_ft_op (solver.py:571-577).
 *                 g = -i alpha_i / (|k|^2 - alpha); no 1/N (the inverse mmx_fftn scales).
 *   mmx_chi_mix:  u = (a chi_EE0 + b I) x + f_HE chi_HE0 d, w = f_EH chi_EH0 x + f_HH chi_HH0 d per voxel, the four
 *                 blocks [9][N] (row-major 3x3) stored at alpha0; coef = the complex pairs (a, b, f_EH, f_HE, f_HH)
 *                 in FP64 (host memory).  Replaces the mul / add steps of chi_op and the rescaling of
 *                 __update_operators (solver.py:514-528).
 *   mmx_axpby:    out = a x + b y (nwords complex words).
 */
int mmx_curl_ft(mmx_plan* plan, const void* F, void* out, void* stream);
int mmx_green_ft(mmx_plan* plan, void* F, double alpha_re, double alpha_im, void* stream);
int mmx_chi_mix(const void* x, const void* d, const void* chi_ee, const void* chi_eh, const void* chi_he,
                const void* chi_hh, const double* coef, void* u, void* w, int64_t nvox, int precision, void* stream);
int mmx_axpby(void* out, const void* x, const void* y, double a_re, double a_im, double b_re, double b_im,
              int64_t nwords, int precision, void* stream);

/*
 * The magnetic iteration on the device: niter iterations of Solution.__iter__ (solver.py:1049-1098) with the
 * magnetic chi_op (solver.py:531-552), the same composition as the kernels above, but with alpha read from and the
 * accept / reject (solver.py:1077-1096) and stop rules (solver.py:81-83) taken in the mmx_rhs_state `st`, so that a
 * chunk of iterations needs no host round trip.  An iteration after which the stop rule fails leaves the state and E
 * unchanged.  `plan`: 1 component, batch 1, the grid's k-vectors set.  use_graph != 0 replays the chunk from a CUDA
 * graph captured on the first call with these buffers and niter.  All buffers [3][N] (blocks [9][N]) in the plan's
 * precision.
 */
typedef struct mmx_magnetic_buffers {
  void* E;            /* the field (times k0^2), updated in place */
  const void* src;    /* normalised source s'0 at alpha0 */
  const void* chi_ee; /* the four susceptibility blocks at alpha0, [9][N] each */
  const void* chi_eh;
  const void* chi_he;
  const void* chi_hh;
  void* work[7];      /* scratch, [3][N] each */
} mmx_magnetic_buffers;
int mmx_magnetic_iterate(mmx_plan* plan, const mmx_magnetic_buffers* buffers, mmx_rhs_state* st, int niter,
                         int use_graph, void* stream);

/*
 * The alpha objective of the preconditioner for a scalar permittivity (replaces the full-grid host evaluation in
 * Solution.__prepare_preconditioner, solver.py:392-401): out_dev[0..1] = min, max over the nvox voxels of
 * (ab^2 - 2 round(x ab)) + p, where xp holds the pairs (x, p) = (Re eps, Re(conj(eps) eps)) in FP64 on the device.
 * This is the host expression |ab|^2 - (conj(eps) ab + eps conj(ab)) + conj(eps) eps (whose imaginary part is zero for
 * real ab) evaluated with explicitly rounded operations, so the largest singular value sqrt(max |.|) / |beta| equals
 * the host's bit for bit.  Uses the plan's scratch.
 */
int mmx_scalar_sigma(mmx_plan* plan, const void* xp, int64_t nvox, double ab, double* out_dev, void* stream);

/*
 * The susceptibility at the preconditioner's alpha from a permittivity already on the device (replaces the host
 * array expression of Solution.__prepare_preconditioner, solver.py:480-484, chi = eps i / (alpha_i beta) - i alpha /
 * alpha_i I):  chi[r][v] = s eps[r][v] - (r on the diagonal ? d : 0) for the m = 1 or 9 row-major entries of a
 * complex128 matrix field eps [m][nvox]; chi is written in `precision` (complex64 or complex128), s and d in FP64.
 */
int mmx_chi_from_eps(const void* eps, int m, int64_t nvox, double s_re, double s_im, double d_re, double d_im,
                     void* chi, int precision, void* stream);

/*
 * mmx_fftn without a plan and without any device allocation: the same transform as mmx_fftn (forward unscaled,
 * inverse scaled by 1/N) over the `ndim` grid axes `shape` of `nbatch` contiguous fields of the given precision.
 * No counterpart in the reference (which always allocates through its backend).  For callers that must not let a
 * library allocate or free device memory: applications that place every buffer through their own pool or fixed
 * memory plan (a serving process with a set memory budget, a framework's caching allocator), where a stray
 * cudaMalloc can fail on a fully committed GPU and a cudaFree stalls the whole device while other streams run.
 * Limits: every axis length at most 4096 and factorisable into 2, 3, 5, 7, 11, 13 (longer axes are rejected with
 * MMX_ERR_UNSUPPORTED).  The twiddle scratch is one 192 KiB __device__ array shared by all calls in the process:
 * calls that overlap on the GPU race; the first call on a device looks up that array's address and should be made
 * before any stream capture.
 */
int mmx_fftn_noalloc(int ndim, const int64_t* shape, const void* in, void* out, int64_t nbatch, int inverse,
                     int precision, void* stream);

/*
 * Scattering-matrix mode synthesis and detection (replaces the spectrum assignment of srcvec2freespace,
 * matrix.py:528-610, and the spectrum lookup of detfield2detvec, matrix.py:685-755).  A row is one
 * transverse plane of `row_len` complex words (precision MMX_C64 | MMX_C128); idx[nmodes] (device, int64) holds the
 * spectrum position of every propagating mode.
 *   mmx_mode_scatter: out[r][idx[m]] = coef[r][m] for r < nrows (the other words of `out` are left as they are);
 *   mmx_mode_gather:  out[r][m] = in[r][idx[m]].
 * conj = 1 conjugates each word on the way.  Positions outside [0, row_len) are skipped (scatter) or read as 0
 * (gather).  The transverse transforms between them are mmx_fftn calls on a plan of the transverse shape.
 */
int mmx_mode_scatter(const void* coef, const int64_t* idx, int64_t nmodes, int64_t nrows, int64_t row_len, int conj,
                     void* out, int precision, void* stream);
int mmx_mode_gather(const void* in, const int64_t* idx, int64_t nmodes, int64_t nrows, int64_t row_len, int conj,
                    void* out, int precision, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MACROMAX_B200_H */
