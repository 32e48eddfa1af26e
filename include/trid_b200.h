/*
 * tridsolver_b200 -- public C ABI of the scalar batched tridiagonal solver
 * (libtridb200.so).
 *
 * Drop-in for the reference's strided-batch API:
 *   scalar/include/trid_cpu.h:53-82   (9-argument form; declared here over
 *                                      DEVICE pointers, one B200 GPU)
 *   scalar/include/trid_cuda.h:44-80  (the 11-argument GPU form with
 *                                      `int *opts, int sync` is exported under
 *                                      the same names by the companion library
 *                                      libtridb200_cudacompat.so, see
 *                                      include/trid_b200_cudacompat.h)
 *   scalar/include/trid_common.h:65-76 (tridStatus_t, same values)
 *
 * Semantics (same as the reference):
 *   - a, b, c, d, u are arrays of shape dims[0..ndim-1] (dims[0] fastest),
 *     padded to pads[0..ndim-1]: element (i0,i1,...) is at
 *     i0 + pads[0]*(i1 + pads[1]*(i2 + ...)).
 *   - One independent system per line along axis `solvedim`:
 *       a_i x_{i-1} + b_i x_i + c_i x_{i+1} = d_i.
 *     a[0] and c[n-1] of every system are never read.
 *   - Non-Inc: the solution overwrites d; u is not used (may be NULL).
 *     Inc:     u += solution; d is left unmodified.
 *   - dims/pads are HOST arrays; a..u are DEVICE pointers (cudaMalloc or
 *     managed memory) aligned to their element size.
 *   - Work is enqueued on the calling thread's stream (tridSetStream, default
 *     the legacy default stream) and the call returns without synchronising.
 *   - Solves that need device scratch (systems too long for one pass, which
 *     are solved in blocks; method 1; the variable-length batch; the block
 *     solver; ADI without a work buffer) take it from a buffer the library
 *     keeps per device and stream, grown on demand (a growing call waits for
 *     that stream's queued work), so calls on different streams or threads
 *     may run concurrently.  A call made while its stream is being captured
 *     into a CUDA graph allocates and frees its scratch in stream order
 *     instead (graph memory nodes), so a captured call needs no earlier
 *     warm-up call and the graph holds no pointer to the kept buffers.
 *     tridReleaseScratch frees the kept buffers.
 *
 * Differences from the reference, all on error paths: invalid arguments
 * return TRID_STATUS_INVALID_VALUE instead of printing and calling exit()
 * (trid_cuda.cu:209-219); a failed launch returns
 * TRID_STATUS_EXECUTION_FAILED instead of aborting; ndim may be 1..8 on
 * every axis (the reference CPU path assumes 3, its GPU x-path needs
 * pads[i>=1] == dims[i]).
 */
#ifndef TRID_B200_H
#define TRID_B200_H

#ifdef __cplusplus
#define TRID_EXTERN_C extern "C"
#else
#define TRID_EXTERN_C
#endif

#define TRID_B200_MAXDIM 8

/* scalar/include/trid_common.h:65-76 -- same names and values. */
typedef enum {
  TRID_STATUS_SUCCESS = 0,
  TRID_STATUS_NOT_INITIALIZED = 1,
  TRID_STATUS_ALLOC_FAILED = 2,
  TRID_STATUS_INVALID_VALUE = 3,
  TRID_STATUS_ARCH_MISMATCH = 4,
  TRID_STATUS_MAPPING_ERROR = 5,
  TRID_STATUS_EXECUTION_FAILED = 6,
  TRID_STATUS_INTERNAL_ERROR = 7,
  TRID_STATUS_MATRIX_TYPE_NOT_SUPPORTED = 8,
  TRID_STATUS_ZERO_PIVOT = 9
} tridStatus_t;

/* ---- strided batch: replaces trid_cpu.h:53-60 (tridS/DmtsvStridedBatch) ---- */
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatch(const float *a, const float *b, const float *c,
                                                 float *d, float *u, int ndim, int solvedim,
                                                 int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatch(const double *a, const double *b,
                                                 const double *c, double *d, double *u, int ndim,
                                                 int solvedim, int *dims, int *pads);

/* ---- Inc variants: replace trid_cpu.h:74-82 (tridS/DmtsvStridedBatchInc) ---- */
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchInc(const float *a, const float *b,
                                                    const float *c, float *d, float *u, int ndim,
                                                    int solvedim, int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchInc(const double *a, const double *b,
                                                    const double *c, double *d, double *u,
                                                    int ndim, int solvedim, int *dims, int *pads);

/* ---- complex element types: the forms the reference declares but leaves
 *      commented out (trid_cuda.h:39-52; trid_cuda.cu:546-600,
 *      tridCmtsvStridedBatch / tridZmtsvStridedBatch and their Inc forms),
 *      with the live 9-argument signature above.  Elements are interleaved
 *      (re, im) pairs -- the layout of cuComplex / cuDoubleComplex,
 *      std::complex and C99 _Complex -- aligned to their size (8 / 16 bytes).
 *      Same algorithm in complex arithmetic, no pivoting: the rows must be
 *      safe for Gaussian elimination without pivoting (e.g. diagonally
 *      dominant in modulus).  These and the Mixed forms below choose their
 *      kernels by length and axis alone (tridSetMethod and the tuning table
 *      apply to the real forms). ---- */
typedef struct {
  float re, im;
} tridComplexF;
typedef struct {
  double re, im;
} tridComplexD;
TRID_EXTERN_C tridStatus_t tridCmtsvStridedBatch(const tridComplexF *a, const tridComplexF *b,
                                                 const tridComplexF *c, tridComplexF *d,
                                                 tridComplexF *u, int ndim, int solvedim,
                                                 int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridCmtsvStridedBatchInc(const tridComplexF *a, const tridComplexF *b,
                                                    const tridComplexF *c, tridComplexF *d,
                                                    tridComplexF *u, int ndim, int solvedim,
                                                    int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridZmtsvStridedBatch(const tridComplexD *a, const tridComplexD *b,
                                                 const tridComplexD *c, tridComplexD *d,
                                                 tridComplexD *u, int ndim, int solvedim,
                                                 int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridZmtsvStridedBatchInc(const tridComplexD *a, const tridComplexD *b,
                                                    const tridComplexD *c, tridComplexD *d,
                                                    tridComplexD *u, int ndim, int solvedim,
                                                    int *dims, int *pads);

/* ---- FP32 storage, FP64 arithmetic (no reference counterpart): the
 *      arguments of tridSmtsvStridedBatch[Inc]; every element is widened to
 *      double on load, the solve runs in double and each result is rounded to
 *      float once (Inc: u = float(double(u) + x)), so the FP32 result is the
 *      correctly rounded FP64 solution up to the FP64 solve's own error. ---- */
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchMixed(const float *a, const float *b,
                                                      const float *c, float *d, float *u,
                                                      int ndim, int solvedim, int *dims,
                                                      int *pads);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchMixedInc(const float *a, const float *b,
                                                         const float *c, float *d, float *u,
                                                         int ndim, int solvedim, int *dims,
                                                         int *pads);

/* ---- per-array pads: replace trid_cuda.h:61-67 / :78-84
 *      (tridDmtsvStridedBatchPadded[Inc]); float forms are additions.
 *      opts is an optional algorithm hint (may be NULL); sync=1 waits for the
 *      solve to finish before returning. ---- */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchPadded(
    const double *a, const int *a_pads, const double *b, const int *b_pads, const double *c,
    const int *c_pads, double *d, const int *d_pads, double *u, const int *u_pads, int ndim,
    int solvedim, int *dims, int *opts, int sync);
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchPaddedInc(
    const double *a, const int *a_pads, const double *b, const int *b_pads, const double *c,
    const int *c_pads, double *d, const int *d_pads, double *u, const int *u_pads, int ndim,
    int solvedim, int *dims, int *opts, int sync);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchPadded(
    const float *a, const int *a_pads, const float *b, const int *b_pads, const float *c,
    const int *c_pads, float *d, const int *d_pads, float *u, const int *u_pads, int ndim,
    int solvedim, int *dims, int *opts, int sync);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchPaddedInc(
    const float *a, const int *a_pads, const float *b, const int *b_pads, const float *c,
    const int *c_pads, float *d, const int *d_pads, float *u, const int *u_pads, int ndim,
    int solvedim, int *dims, int *opts, int sync);

/* ---- adjoint (no reference counterpart) ----------------------------------
 * Reverse-mode derivative of tridXmtsvStridedBatch.  For x = A^{-1} d (the
 * systems of the forward call) and a cotangent w = dL/dx, computes
 *   g = A^{-T} w,  dd = g,  da_i = -g_i x_{i-1},  db_i = -g_i x_i,
 *   dc_i = -g_i x_{i+1}   (da_0 = dc_{n-1} = 0: those entries are unused).
 * u is the forward solution x.  Every array has the layout of dims/pads (one
 * pads array for all).  Outputs are overwritten; any of da, db, dc, dd may be
 * NULL.  Outputs must not alias a, b, c or u (dd may alias w).  Device
 * pointers, enqueued on the calling thread's stream.  The transposed system
 * (sub-diagonal c_{i-1}, super-diagonal a_{i+1}) is solved in place by the
 * partitioned-Thomas kernels, gradients formed in the same pass. */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchAdjoint(const double *a, const double *b,
                                                        const double *c, const double *u,
                                                        const double *w, double *da, double *db,
                                                        double *dc, double *dd, int ndim,
                                                        int solvedim, int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchAdjoint(const float *a, const float *b,
                                                        const float *c, const float *u,
                                                        const float *w, float *da, float *db,
                                                        float *dc, float *dd, int ndim,
                                                        int solvedim, int *dims, int *pads);

/* ---- out-of-place forward solve (no reference counterpart) ----------------
 * x = A^{-1} d with d left intact (one pads array for every operand; x may
 * be d, which is then the ordinary in-place solve).  Saves the copy of d a
 * caller that must keep its right-hand side (an autograd forward) would
 * otherwise make: on axis 0 up to 4096 rows the one-CTA kernel writes x
 * directly, elsewhere the blocked partition reads d and writes x. */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchOut(const double *a, const double *b,
                                                    const double *c, const double *d, double *x,
                                                    int ndim, int solvedim, int *dims, int *pads);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchOut(const float *a, const float *b, const float *c,
                                                    const float *d, float *x, int ndim,
                                                    int solvedim, int *dims, int *pads);

/* ---- forward solve + adjoint in one call (no reference counterpart) -------
 * x = A^{-1} d and, for the cotangent w = dL/dx, the gradients of the
 * adjoint above at that x (dd = A^{-T} w, da, db, dc), in one call.  For
 * solvedim 0 and n <= 4096 one kernel does both (every input read once,
 * method 6 below); otherwise the forward solve and the adjoint run one
 * after the other.  x
 * may alias d and dd may alias w; no other output may alias an input. */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchFwdAdj(const double *a, const double *b,
                                                       const double *c, const double *d,
                                                       const double *w, double *x, double *da,
                                                       double *db, double *dc, double *dd,
                                                       int ndim, int solvedim, int *dims,
                                                       int *pads);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchFwdAdj(const float *a, const float *b,
                                                       const float *c, const float *d,
                                                       const float *w, float *x, float *da,
                                                       float *db, float *dc, float *dd, int ndim,
                                                       int solvedim, int *dims, int *pads);

/* Systems split along the solve dimension across ranks (one slab of rows
 * per rank, in rank order): the two device-side phases of the reference's
 * tridDmtsvStridedBatchMPI / tridDmtsvStridedBatchIncMPI
 * (scalar/include/trid_mpi_cuda.hpp:51-80, implementation
 * scalar/src/cuda/trid_cuda_mpi.cu:473-583).  The exchange between them is
 * the caller's -- an all-gather of `bnd` over the ranks of the solve
 * dimension (tridsolver_b200/mpi.py does it over torch.distributed):
 *   SplitReduce : this rank's slab (dims/pads are the local extents; at least
 *                 2 rows along solvedim) reduced to six FP64 numbers per
 *                 system, bnd laid out [6][nsys] (nsys = product of the other
 *                 dims, systems in the order of the strided-batch solve);
 *   SplitFinish : bnd_all = every rank's bnd, [nranks][6][nsys] in rank
 *                 order; solves this rank's slab (into d, or added into u
 *                 when inc != 0, d then left as it was).  a of the first
 *                 rank's first row and c of the last rank's last row are
 *                 ignored, as in the single-GPU solve.
 * Errors as the strided-batch solve; both are stream-ordered. */
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchSplitReduce(const double *a, const double *b,
                                                            const double *c, const double *d,
                                                            int ndim, int solvedim,
                                                            const int *dims, const int *pads,
                                                            double *bnd);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchSplitReduce(const float *a, const float *b,
                                                            const float *c, const float *d,
                                                            int ndim, int solvedim,
                                                            const int *dims, const int *pads,
                                                            double *bnd);
TRID_EXTERN_C tridStatus_t tridDmtsvStridedBatchSplitFinish(const double *a, const double *b,
                                                            const double *c, double *d, double *u,
                                                            int ndim, int solvedim,
                                                            const int *dims, const int *pads,
                                                            const double *bnd_all, int nranks,
                                                            int rank, int inc);
TRID_EXTERN_C tridStatus_t tridSmtsvStridedBatchSplitFinish(const float *a, const float *b,
                                                            const float *c, float *d, float *u,
                                                            int ndim, int solvedim,
                                                            const int *dims, const int *pads,
                                                            const double *bnd_all, int nranks,
                                                            int rank, int inc);

/* ---- variable-length packed batch (no reference counterpart) --------------
 * nsys independent systems packed back to back: system s occupies rows
 * [offsets[s], offsets[s+1]) of a, b, c, d (unit stride); offsets is a DEVICE
 * array of nsys+1 int64 values and total = offsets[nsys] (the number of
 * rows, passed so that the call needs no device-to-host read).  Each system's
 * first a and last c are never read.  The solution overwrites d.  Systems of
 * up to 8192 rows: three short preparation launches sort them into
 * length-bucketed work queues (up to 256 rows, one warp each; 257 .. 4096
 * rows, one CTA of ceil(n/512) warps each, by bucket; 4097 .. 8192 rows, one
 * CTA each), each served by persistent CTAs.  Malformed offsets and longer
 * systems are skipped and reported by tridGetDeviceErrors (bits 4 and 8).
 * Offsets must increase monotonically: where they do not, valid-looking
 * systems may overlap (each is solved in place in turn, in no fixed order);
 * no work table can overflow, whatever the offsets hold. */
TRID_EXTERN_C tridStatus_t tridDmtsvVarlenBatch(const double *a, const double *b, const double *c,
                                                double *d, const long long *offsets,
                                                long long nsys, long long total);
TRID_EXTERN_C tridStatus_t tridSmtsvVarlenBatch(const float *a, const float *b, const float *c,
                                                float *d, const long long *offsets,
                                                long long nsys, long long total);

/* Allocation-free FP64 variant of tridDmtsvVarlenBatch; it has no
 * counterpart in the reference.  For callers that cannot allocate device
 * memory -- code running under another component's allocator or memory budget
 * (a driver allocation would take memory the pool reserved, or fail) and
 * latency-critical loops that cannot absorb the device synchronisation of
 * cudaMalloc/cudaFree.  Same arguments and result as tridDmtsvVarlenBatch,
 * but every scratch byte comes from one fixed 32 MiB array per device that
 * the library holds from load to process exit; no call allocates.
 * Limit: the work space must fit in 32 MiB, roughly 40*nsys bytes plus
 * alignment (about 830,000 systems, whatever their total length); larger
 * problems return TRID_STATUS_INVALID_VALUE and should use
 * tridDmtsvVarlenBatch.
 * The first call on each device looks up the array's device address (a
 * runtime symbol query, no allocation) with that device current; make that
 * first call before any stream capture.  Every call uses the same array and
 * leaves its contents behind (the next call clears what must start at zero),
 * so calls that overlap on the GPU -- concurrent streams or threads on one
 * device -- race and must be serialised by the caller.  Malformed offsets
 * and over-long systems are skipped as in tridDmtsvVarlenBatch and recorded
 * in an error word inside the same array, which tridGetDeviceErrors reads
 * and clears together with the library's word (bits 4 and 8; that call
 * allocates nothing either).  No kernel of the solve waits on another CTA. */
TRID_EXTERN_C tridStatus_t tridDmtsvVarlenBatchNoAlloc(const double *a, const double *b,
                                                       const double *c, double *d,
                                                       const long long *offsets, long long nsys,
                                                       long long total);

/* ---- ADI heat diffusion (the reference app apps/adi/src/adi_orig.c:147-240,
 *      adi_cuda.cu:285-329, rebuilt around generated coefficients) ----------
 * Grid nx*ny*nz (x fastest, each extent 1..512).  Interior points get the
 * tridiagonal row (a, b, c) along every axis, face points the identity row;
 * the step RHS is lambda*(sum of the 6 neighbours - 6u) on interior points, 0
 * on faces (the reference app uses a = c = -lambda/2, b = 1 + lambda).
 *
 * tridXadiSteps: nsteps steps u <- u + Z^{-1} Y^{-1} X^{-1} rhs(u), three
 *   launches per step (stencil fused into the x solve, u += in the z solve).
 *   work holds 2*nx*ny*nz elements (NULL = library scratch).
 * tridXadiSolve: one axis solve out = T^{-1} rhs with T the generated
 *   operator along `axis` (0, 1, 2); stencil=1 (axis 0 only) takes u in rhs
 *   and solves for the step RHS; transpose=1 solves with T^T (adjoint);
 *   inc=1 (axes 1, 2) adds the solution into out.
 * tridDadiLaplacianT: out += lambda * L^T g (L the interior-masked
 *   7-point Laplacian): the stencil's adjoint.
 * tridDadiStepVjp: the rest of one step's adjoint in one pass.  Given the
 *   step's input u, its parts du1 = X^{-1} lambda L u, du2 = Y^{-1} du1,
 *   du3 = Z^{-1} du2 and the transposed solves g3 = Z^{-T} ubar,
 *   g2 = Y^{-T} g3, g1 = X^{-T} g2: ubar += lambda L^T g1 (the cotangent of
 *   u) and *lbar += <g1, L u> - <g1, X' du1> - <g2, Y' du2> - <g3, Z' du3>,
 *   X' = dX/dlambda (interior rows (da, db, dc): (-1/2, 1, -1/2) for the
 *   reference coefficients, (-1, 2, -1) for the plain ones).  lbar is
 *   one device double, accumulated in place; the sum is formed in a fixed
 *   order (same result on every run). */
TRID_EXTERN_C tridStatus_t tridDadiSteps(double *u, double *work, int nx, int ny, int nz,
                                         int nsteps, double lambda, double a, double b, double c);
TRID_EXTERN_C tridStatus_t tridSadiSteps(float *u, float *work, int nx, int ny, int nz, int nsteps,
                                         float lambda, float a, float b, float c);
TRID_EXTERN_C tridStatus_t tridDadiSolve(const double *rhs, double *out, int nx, int ny, int nz,
                                         int axis, int stencil, int transpose, int inc,
                                         double lambda, double a, double b, double c);
TRID_EXTERN_C tridStatus_t tridSadiSolve(const float *rhs, float *out, int nx, int ny, int nz,
                                         int axis, int stencil, int transpose, int inc,
                                         float lambda, float a, float b, float c);
TRID_EXTERN_C tridStatus_t tridDadiLaplacianT(const double *g, double *out, int nx, int ny, int nz,
                                              double lambda);
TRID_EXTERN_C tridStatus_t tridDadiStepVjp(const double *u, const double *du1, const double *du2,
                                           const double *du3, const double *g1, const double *g2,
                                           const double *g3, double *ubar, int nx, int ny, int nz,
                                           double lambda, double da, double db, double dc,
                                           double *lbar);

/* ---- replaces trid_cuda.h:44 (a no-op in the reference, trid_cuda.cu:612) ---- */
TRID_EXTERN_C void initTridMultiDimBatchSolve(int ndim, int *dims, int *pads);

/* ---- extensions (no reference counterpart) -------------------------------- */

/* Stream used by every call made from the calling thread (a cudaStream_t;
 * NULL = legacy default stream). */
TRID_EXTERN_C tridStatus_t tridSetStream(void *stream);
TRID_EXTERN_C void *tridGetStream(void);

/* Free the scratch buffers the library keeps for the current device (every
 * stream's), after waiting for the device to finish its queued work.  Call
 * it when no other thread is calling into the library on this device; the
 * next solve that needs scratch allocates again. */
TRID_EXTERN_C tridStatus_t tridReleaseScratch(void);

/* Human-readable name of a status code. */
TRID_EXTERN_C const char *tridGetStatusString(tridStatus_t status);

/* Algorithm selection for the scalar solves (autotuner hook).
 *   method 0 = automatic (tuning table, then built-in heuristics)
 *   method 1 = Thomas, one thread per system, c'/d' in library scratch
 *              (systems longer than 32*chunk rows are cut into blocks of
 *              32*chunk rows by methods 2/3: block reduction, block system
 *              solved recursively, block finish)
 *   method 2 = partitioned Thomas: per-thread chunks of `chunk` rows reduced to
 *              a 64-row interface system solved by warp shuffles (PCR); the
 *              rows are staged by TMA (bulk tensor copies) when the layout
 *              allows.  On strided axes a tile of 128 bytes of systems (16
 *              FP64 / 32 FP32, the default up to 256 rows) streams through
 *              one persistent CTA per SM, the next tile's copy in flight
 *              while the current one is solved
 *   method 3 = method 2 with plain loads only
 *   methods 4 and 5 are not used (INVALID_VALUE)
 *   method 6 = axis 0: one CTA per system, one block of 32*chunk rows per
 *              warp (chunk 4, 8 or 16; up to 4096 rows)
 *              (method 6 acts as method 3 on the other axes and past 4096
 *              rows; by default axis-0 systems of 513..4096 rows take
 *              method 6 with chunk 16, as do the adjoint and the forward +
 *              adjoint call from 65 rows)
 *   chunk      : rows per thread for methods 2/3 (2, 4, 8 or 16; 0 = automatic)
 *   sys_per_cta: systems per CTA for methods 2/3 on strided axes (4, 8, 16 or
 *                32; 0 = auto; 32 applies to the FP32 streamed tiles, and
 *                the plain-load kernels cap it at 16)
 * Applies to calls from the calling thread. */
TRID_EXTERN_C tridStatus_t tridSetMethod(int method, int chunk, int sys_per_cta);

/* Error bits recorded on the current device by kernels whose bounded waits
 * gave up (1 = a TMA/mbarrier wait timed out; 2 = a bulk-copy shared-memory
 * operand was misaligned and the copy was skipped; 4 = malformed varlen
 * offsets; 8 = a varlen system longer than supported); reading clears them.
 * Covers the allocation-free varlen solve's word too.  Allocates nothing;
 * blocks until the device is idle. */
TRID_EXTERN_C tridStatus_t tridGetDeviceErrors(unsigned *flags);

/* Load an autotuning table written by tridsolver_b200.autotune (text lines
 * "<dtype> <axis class> <nmax> <method> <chunk> <sys_per_cta>", dtype f32 or
 * f64, axis class as in tridQueryMethod; class 4 lines "<dtype> 4 <nmax> 2
 * <chunk> 0" set the variable-length batch's length buckets: systems of up
 * to nmax rows take `chunk` rows per lane, 2 up to at most 64 rows, 4 up to
 * at most 128, else 8); NULL clears it.  Process-wide.
 * The first solve of a process also loads the file named by the environment
 * variable TRID_B200_TUNING, when set. */
TRID_EXTERN_C tridStatus_t tridLoadTuningTable(const char *path);

/* The method/chunk/sys_per_cta the dispatcher would use for a problem:
 * dtype_bytes 4 or 8; axis class 0 = solve along axis 0 (unit stride),
 * 1 = strided solve with a row stride of at most 64 KiB, 2 = at most 1 MiB,
 * 3 = larger stride, 4 = a system of n rows in a variable-length batch
 * (method 2, chunk = its rows per lane). */
TRID_EXTERN_C tridStatus_t tridQueryMethod(int dtype_bytes, int axis, int n, int *method,
                                           int *chunk, int *sys_per_cta);

#endif /* TRID_B200_H */
