/*
 * seldon_b200.h -- C ABI of libseldon_b200.so, the B200 (sm_100a) engine
 * behind Seldon's sparse Krylov path.
 *
 * Every entry point replaces one routine of the reference (Seldon, a
 * header-only C++ template library).  The reference "interface" is a set of
 * free-function overloads resolved by argument-dependent lookup; the citation
 * beside each declaration names the overload it stands in for (file:line in
 * the Seldon tree).  include/SeldonB200.hxx maps Seldon's C++ templates onto
 * these functions, so a Seldon user changes only an allocator argument.
 *
 * Conventions
 *   - Sizes and CSR indices are int32, as in Seldon (Matrix_Sparse.hxx:60-64).
 *   - Vector arguments are DEVICE pointers unless the name says _host.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default).
 *   - Every function returns an int status: SB2_OK (0) or a negative SB2_ERR_*
 *     code.  Nothing throws, nothing aborts: a host allocation that fails
 *     inside a call gives SB2_ERR_NO_MEMORY, any other C++ exception raised
 *     inside it SB2_ERR_HOST.  Solver convergence/breakdown is
 *     NOT a status: it is reported in sb2_iter_result.error_code exactly as
 *     Seldon's Iteration::ErrorCode() (Iterative.cxx:344-354).
 *   - Device-side waits (grid barriers of the fused solvers) are bounded; a
 *     wait that runs out ends the kernel and the call returns SB2_ERR_TIMEOUT.
 *   - Threads: calls from several host threads, each on its own stream, may
 *     share a matrix handle.  Its lazily built members (transpose, diagonal,
 *     FP32 copy, cluster plan) are built under the handle's lock and
 *     published only when complete.  Solver work vectors come from a
 *     stream-ordered pool, and reduction scratch is kept per (device,
 *     stream).  A preconditioner or batch handle holds work arrays of its
 *     own (the SOR and ILUT sweeps' temporary, the batch residuals): one
 *     stream at a time, as Seldon's objects are used by one thread at a time.
 *     sb2_cg_noalloc shares one scratch per device (see its declaration).
 *     Destroying a handle that a call still uses is the caller's error.
 */
#ifndef SELDON_B200_H
#define SELDON_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define SB2_OK 0
#define SB2_ERR_INVALID_VALUE -1 /* bad sizes / null pointers / aliasing */
#define SB2_ERR_NO_MEMORY -2     /* a device or host allocation failed */
#define SB2_ERR_CUDA -3          /* any other CUDA runtime error */
#define SB2_ERR_TIMEOUT -4       /* a bounded device-side wait ran out */
#define SB2_ERR_INVALID_CSR -5   /* CSR invariants violated (validator) */
#define SB2_ERR_NOT_SUPPORTED -6 /* option combination not implemented */
#define SB2_ERR_HOST -7          /* any other host-side failure */

/* Human-readable text for a status code (static storage). */
const char* sb2_status_string(int status);

/* Library version, e.g. 10000 for 1.0.0. */
int sb2_version(void);

/* ------------------------------------------------------------ device memory */

/* Device buffers for callers that do not link the CUDA runtime themselves
 * (the CudaAlloc allocator of SeldonB200.hxx).  They stand in for the
 * allocator concept's allocate/deallocate/memorycpy (share/Allocator.hxx:
 * 31-48, share/Allocator.cxx:33-65) on device memory.
 *   sb2_device_alloc  cudaMalloc of `bytes` (bytes == 0 gives NULL)
 *   sb2_device_free   cudaFree (NULL is a no-op); arrays that sb2_coo_to_csr
 *                     returned go back to the library's memory pool, after
 *                     the device has finished its work, as cudaFree waits
 *   sb2_memcpy        copy `bytes` between host and/or device memory
 *                     (unified addressing decides the direction), on
 *                     `stream`; returns after the copy has completed
 *   sb2_stream_sync   wait for all work queued on `stream` */
int sb2_device_alloc(size_t bytes, void** out);
int sb2_device_free(void* p);
int sb2_memcpy(void* dst, const void* src, size_t bytes, void* stream);
int sb2_stream_sync(void* stream);

/* ------------------------------------------------------------ CSR handle */

/* Opaque device CSR matrix (device copies of ptr_/ind_/data_ plus the
 * row-block partition the SpMV kernels use). */
typedef struct sb2_csr sb2_csr;

/* Create a device matrix from arrays in Seldon's layout (all three in host
 * memory, or all three in device memory).
 *   m, n, nnz          sizes (nnz = ptr[m])
 *   ptr[m+1], ind[nnz], val[nnz]   Seldon's ptr_, ind_, data_
 *   symmetric_upper    0: Matrix<double, General, RowSparse>
 *                      1: Matrix<double, Symmetric, RowSymSparse>: only the
 *                         upper triangle (diagonal included) is given
 *                         (Matrix_SymSparse.cxx:1031-1032)
 *   validate           1: check ptr monotone, ptr[0]=0, ptr[m]=nnz,
 *                         0<=ind<n (and ind>=row for symmetric_upper), as
 *                         SELDON_CHECK_DIMENSIONS does (Matrix_Sparse.cxx:118-170)
 * The arrays are copied; the caller keeps ownership.  They may also be
 * device arrays (sb2_coo_to_csr's output): those are read back to the host,
 * where the validator and the slice layout are built.
 * Replaces the constructor Matrix_Sparse(i, j, values, ptr, ind)
 * (Matrix_Sparse.cxx:105-180) and SetData (Matrix_Sparse.cxx:305-415). */
int sb2_csr_create(int m, int n, int nnz, const int* ptr, const int* ind,
                   const double* val, int symmetric_upper, int validate,
                   sb2_csr** out);

/* Release a matrix (Matrix_Sparse::~Matrix_Sparse, Matrix_Sparse.cxx:206). */
int sb2_csr_destroy(sb2_csr* A);

/* Sizes: rows, columns, stored nonzeros (upper part for symmetric) and the
 * nonzeros of the full operator.  (GetM/GetN/GetNonZeros, Matrix_Sparse.hxx:101-106) */
int sb2_csr_info(const sb2_csr* A, int* m, int* n, int* nnz_stored,
                 int* nnz_full);

/* Copy the stored arrays back to host buffers (ptr[m+1], ind[nnz_stored],
 * val[nnz_stored]); any pointer may be NULL. */
int sb2_csr_download(const sb2_csr* A, int* ptr, int* ind, double* val);

/* Assemble CSR arrays on the device from coordinate triplets, as
 * ConvertMatrix_from_Coordinates does (Matrix_Conversions.cxx:1291-1334 for
 * RowSparse, 1397-1467 for RowSymSparse; ReadText and FillRand reach it too).
 *   row, col, val      DEVICE arrays of nnz triplets, indices from `index`
 *   m_min, n_min       the target matrix's current size (GetM/GetN)
 *   symmetric_upper    0: RowSparse.  m = max(largest row + 1, m_min),
 *                         n = max(largest column + 1, n_min); an empty input
 *                         gives max(1, m_min) x max(1, n_min)
 *                      1: RowSymSparse.  Entries below the diagonal are
 *                         dropped; m = n = largest row (of all entries) + 1;
 *                         an empty input gives m_min x m_min with no entries
 *   stream             orders the work; the call returns when it is done
 * Entries come out in stable (row, column) order, duplicates kept, exactly
 * Seldon's order (its merge sort is stable).  *ptr (m+1), *ind and *val_out
 * (*nnz_out entries) are device arrays allocated here: release them with
 * sb2_device_free.  An index below `index` or past INT_MAX-1 gives
 * SB2_ERR_INVALID_VALUE (ReadCoordinateMatrix's IOError,
 * Matrix_Sparse.cxx:1912-1921).  Nothing is returned on error. */
int sb2_coo_to_csr(int nnz, const int* row, const int* col, const double* val,
                   int index, int m_min, int n_min, int symmetric_upper,
                   void* stream, int* m, int* n, int* nnz_out, int** ptr,
                   int** ind, double** val_out);

/* ------------------------------------------------------------ SpMV */

/* y = beta*y + alpha*op(A)*x  with op = A (trans=0) or A^T (trans=1).
 * Seldon semantics: y is scaled by beta even when beta == 0, so a NaN in y
 * stays NaN.  x and y must not overlap.
 * Replaces MltAdd(alpha, M, X, beta, Y) for RowSparse
 * (Functions_MatVect.cxx:398-431), RowSymSparse (:526-564), and
 * MltAdd(alpha, SeldonTrans, M, X, beta, Y) (:729-758; symmetric :915-927). */
int sb2_spmv(const sb2_csr* A, int trans, double alpha, const double* x,
             double beta, double* y, void* stream);

/* y = alpha*op(A)*x, y overwritten (not read).
 * Replaces Mlt(M, X, Y) / Mlt(alpha, M, X, Y) / Mlt(Trans, M, X, Y)
 * (Functions_MatVect.cxx:72-130: Y.Fill(0) then MltAdd(alpha, M, X, 0, Y)). */
int sb2_mlt(const sb2_csr* A, int trans, double alpha, const double* x,
            double* y, void* stream);

/* MltAdd with HOST vectors: x is copied in, y is copied in (beta != 0) and
 * back out, on `stream`; returns after y is back on the host.  For callers
 * whose vectors live in host memory (Seldon's default MallocAlloc). */
int sb2_spmv_host(const sb2_csr* A, int trans, double alpha,
                  const double* x_host, double beta, double* y_host,
                  void* stream);

/* Mlt with HOST vectors: y_host = alpha*op(A)*x_host (y not read).
 * Same reference routine as sb2_mlt (Functions_MatVect.cxx:72-130). */
int sb2_mlt_host(const sb2_csr* A, int trans, double alpha,
                 const double* x_host, double* y_host, void* stream);

/* Mlt over a batch of HOST vectors: y_i = alpha*op(A)*x_i for i < count, with
 * x_host holding count vectors of op(A)'s column size back to back and
 * y_host count vectors of its row size.  The copies in and out and the
 * products are pipelined (copy of x_{i+1}, product i and copy of y_{i-1}
 * overlap); pinned host memory lets the copies run asynchronously.  Returns
 * after every y_i is on the host.  Each y_i is the same bits as sb2_mlt_host
 * on x_i.  No reference counterpart: the reference calls Mlt once per
 * vector (Functions_MatVect.cxx:72-83). */
int sb2_mlt_host_batch(const sb2_csr* A, int trans, double alpha, int count,
                       const double* x_host, double* y_host, void* stream);

/* Device-side condition of the standalone products queued on `stream` so
 * far (the TMA ring engine's bounded waits record it there; the product
 * calls themselves return before their kernels run): *status receives 0
 * (none) or 1 (a bounded wait ran out: the CTA left its share of rows
 * unwritten), and the word is cleared.  Waits for the stream.  No
 * counterpart in the reference. */
int sb2_spmv_status(void* stream, int* status);

/* Product algorithm and launch configuration, chosen by the autotuner; no
 * counterpart in the reference (tuning knobs of this engine).
 *   algo     SB2_SPMV_SELL   binned SELL-32 (thread/warp/CTA per row), default
 *            SB2_SPMV_STREAM row blocks streamed through shared memory
 *            SB2_SPMV_TMA    row blocks in a TMA bulk-copy ring
 *   threads  256 or 512 (TMA kernel), stages 3 or 4 (TMA ring depth) */
#define SB2_SPMV_SELL 0
#define SB2_SPMV_STREAM 1
#define SB2_SPMV_TMA 2
int sb2_spmv_set_config(int algo, int threads, int stages);

/* Measurement of the gather bound of a product: partials[c] (device, one per
 * CTA; *blocks CTAs, at most max_blocks) receive the CTA sums of
 * val[k] * x[ind[k]] (val == NULL: of x[ind[k]]) over k < nnz, all entries
 * in one stream with no rows.  It reads the index and value arrays and
 * gathers x as a CSR product over the same arrays does, so its time bounds
 * from below what any row binning of that product can reach.  ind and val
 * must be 16-byte aligned; ind entries must index x (not checked).  No
 * counterpart in the reference: a measurement kernel the solvers never
 * call. */
int sb2_probe_gather(long long nnz, const int* ind, const double* val, const double* x,
                     double* partials, int max_blocks, int* blocks, void* stream);

/* ------------------------------------------------------------ BLAS-1 (FP64) */
/* All reductions are deterministic: the same n gives the same summation tree
 * on every call and every run. */

/* *result (host) = sum_i x_i*y_i.  DotProd / DotProdConj (real)
 * (Functions_Vector.cxx:330-346, :391-397; cblas_ddot Blas_1.cxx:428-438). */
int sb2_dot(int n, const double* x, const double* y, double* result,
            void* stream);

/* *result (host) = sqrt(sum_i x_i^2).  Norm2 (Functions_Vector.cxx:540-549;
 * cblas_dnrm2 Blas_1.cxx:611-615). */
int sb2_nrm2(int n, const double* x, double* result, void* stream);

/* Device-result forms: write the scalar to device memory, do not synchronize. */
int sb2_dot_device(int n, const double* x, const double* y, double* d_result,
                   void* stream);
int sb2_nrm2_device(int n, const double* x, double* d_result, void* stream);

/* y += alpha*x; no-op when alpha == 0.  Add (Functions_Vector.cxx:85-105;
 * cblas_daxpy Blas_1.cxx:353-365). */
int sb2_axpy(int n, double alpha, const double* x, double* y, void* stream);

/* x *= alpha.  Mlt(alpha, X) (Functions_Vector.cxx:69-74; cblas_dscal
 * Blas_1.cxx:212-216). */
int sb2_scal(int n, double alpha, double* x, void* stream);

/* y = x.  Copy (Functions_Vector.cxx:240-246; cblas_dcopy Blas_1.cxx:282-293). */
int sb2_copy(int n, const double* x, double* y, void* stream);

/* x_i = value.  Vector::Fill / Zero (vector/Vector.cxx:687). */
int sb2_fill(int n, double value, double* x, void* stream);

/* ------------------------------------------------------------ preconditioners */

#define SB2_PRECOND_IDENTITY 0 /* Preconditioner_Base (Iterative.cxx:50-77) */
#define SB2_PRECOND_JACOBI 1   /* z_i = r_i / A(i,i); absent from the reference */
#define SB2_PRECOND_SOR 2      /* SorPreconditioner (Precond_Ssor.cxx:24-90) */
#define SB2_PRECOND_ILUT 3     /* IlutPreconditioning's apply (IlutPreconditioning.cxx) */

typedef struct sb2_precond sb2_precond;

/* kind: SB2_PRECOND_*.  omega, nb_iter, symmetric: SorPreconditioner's
 * SetParameterRelaxation / SetNumberIterations / Init(Un)SymmetricPreconditioning
 * (Precond_Ssor.cxx:36-39; defaults omega=1, nb_iter=1, symmetric=1). */
int sb2_precond_create(const sb2_csr* A, int kind, double omega, int nb_iter,
                       int symmetric, sb2_precond** out);
int sb2_precond_destroy(sb2_precond* M);

/* ILUT preconditioner from a factor computed on the host by Seldon's
 * IlutPreconditioning (FactorizeMatrix / FactorizeSymMatrix, GetIlut):
 *   fptr[n+1], find, fval   the factor's rows in stored order
 *       symmetric = 0: ArrayRowSparse rows: L part (columns < i), then
 *                      1/U(i,i), then the U part (columns > i)
 *                      (SparseSolver.cxx:533-611)
 *       symmetric = 1: ArrayRowSymSparse rows: 1/D(i) first (its index is
 *                      not read), then row i of L^T (columns > i)
 *                      (SparseSolver.cxx:852-882)
 *   perm_row, perm_col      permutation_row / permutation_col (perm_col is
 *                           not read when symmetric)
 *   A                       the system matrix, or NULL: the factor is all
 *                           the apply reads, and the solvers then accept it
 *                           for any matrix of order n
 * Solve / TransSolve (IlutPreconditioning.cxx:329-374) then run on the
 * device as level-scheduled sweeps with the reference's own operation order:
 * z is the reference's z bit for bit.  The arrays are copied.  A factor
 * whose rows break the layout above gives SB2_ERR_INVALID_CSR, a
 * permutation that is not one SB2_ERR_INVALID_VALUE.  The Krylov drivers
 * accept it (device-resident chains around its sweeps, sb2_krylov_set_pcg);
 * sb2_ir_solve does not (SB2_ERR_NOT_SUPPORTED). */
int sb2_precond_create_ilut(const sb2_csr* A, int n, const int* fptr,
                            const int* find, const double* fval,
                            const int* perm_row, const int* perm_col,
                            int symmetric, sb2_precond** out);

/* ILUT factorization on the host, as IlutPreconditioning::FactorizeMatrix
 * computes it for a RowSparse matrix with the unsymmetric algorithm
 * (IlutPreconditioning.cxx:266-323, GetIlut :503-878): the same factor and
 * permutations, bit for bit, for sb2_precond_create_ilut.  Fields follow the
 * reference's setters and defaults (IlutPreconditioning.cxx:27-40):
 *   type             SB2_ILUT (default), SB2_ILU_D or SB2_ILUT_K
 *   fill_level       lfil, the entries kept per part (default 1000000)
 *   additional_fill  ILUT_K: lfil = row length + this (default 1000000)
 *   mbloc            pivots are sought within blocks of mbloc columns
 *                    (default 1000000)
 *   alpha            ILU_D: weight of the dropped sum added to the pivot
 *                    (default 1)
 *   droptol          dropping threshold (default 0.01)
 *   permtol          pivoting threshold (default 0.1) */
#define SB2_ILUT 0
#define SB2_ILU_D 1
#define SB2_ILUT_K 2
typedef struct {
  int type;
  int fill_level;
  int additional_fill;
  int mbloc;
  double alpha;
  double droptol;
  double permtol;
} sb2_ilut_params;

/* The factor of a RowSparse matrix given by HOST arrays (ptr[n+1], ind, val;
 * no repeated column in a row: SB2_ERR_NOT_SUPPORTED) and an ordering perm
 * (FactorizeMatrix's perm; the identity for none).  A row whose entries are
 * all zero gives SB2_ERR_INVALID_VALUE (the reference aborts), and so does
 * an ILUT or ILUT_K fill below 1 for some row (fill_level 0, or
 * additional_fill <= -row length), which keeps no pivot and where the
 * reference writes past the row it resized.  The result
 * is read with sb2_ilut_size / sb2_ilut_arrays (fptr[n+1], find[nnz],
 * fval[nnz], perm_row[n], perm_col[n]) and released with sb2_ilut_destroy. */
typedef struct sb2_ilut sb2_ilut;
int sb2_ilut_factor(int n, const int* ptr, const int* ind, const double* val,
                    const int* perm, const sb2_ilut_params* params,
                    sb2_ilut** out);
/* The symmetric algorithm (SetSymmetricAlgorithm; FactorizeSymMatrix,
 * IlutPreconditioning.cxx:216-263, GetIlut of SymmetricIlutPreconditioning.cxx:
 * 27-346) for a RowSymSparse matrix given by its upper triangle: row i of
 * the factor holds 1/D(i) first, then row i of L^T.  perm_col repeats
 * perm_row. */
int sb2_ilut_factor_sym(int n, const int* ptr, const int* ind,
                        const double* val, const int* perm,
                        const sb2_ilut_params* params, sb2_ilut** out);
int sb2_ilut_size(const sb2_ilut* f, int* n, int* nnz);
int sb2_ilut_arrays(const sb2_ilut* f, int* fptr, int* find, double* fval,
                    int* perm_row, int* perm_col);
int sb2_ilut_destroy(sb2_ilut* f);

/* ILU(0) computed on the device: IlutPreconditioning with
 * SetFactorisationType(ILU_0) and the identity ordering on a RowSparse
 * matrix (GetIlu0, IlutPreconditioning.cxx:1115-1176), or with `modified`
 * MILU_0 (GetMilu0, :1178-1243), row by row in levels of the L pattern,
 * each row in the reference's operation order: the factor is the
 * reference's bit for bit.  A's rows must be sorted by column, without
 * repeats, and hold their diagonal (SB2_ERR_INVALID_CSR otherwise); a zero
 * pivot gives SB2_ERR_INVALID_VALUE (the reference aborts).  The result is an
 * SB2_PRECOND_ILUT preconditioner that keeps no reference to A (as one made
 * by sb2_precond_create_ilut with A == NULL): A may be destroyed after the
 * call, and the solvers take it with any matrix of order n. */
int sb2_precond_create_ilu0(const sb2_csr* A, int modified, void* stream,
                            sb2_precond** out);

/* z = M^{-1} r (Solve) / M^{-T} r (TransSolve).  z and r must not overlap.
 * Precond_Ssor.cxx:62-90: z is zeroed, then SOR type 0 (symmetric), 2
 * (forward, Solve) or 3 (backward, TransSolve). */
int sb2_precond_solve(const sb2_precond* M, const double* r, double* z,
                      void* stream);
int sb2_precond_trans_solve(const sb2_precond* M, const double* r, double* z,
                            void* stream);

/* In-place relaxation on x: SOR(A, X, B, omega, iter, type_ssor) with
 * type_ssor 2 (forward), 3 (backward) or 0 (both), reproducing the
 * sequential sweep order exactly by level scheduling.
 * Relaxation_MatVect.cxx:41-95 (RowSparse), :176-298 (RowSymSparse). */
int sb2_sor(const sb2_csr* A, double* x, const double* b, double omega,
            int iter, int type_ssor, void* stream);

/* ------------------------------------------------------------ iterative solvers */

/* Iteration<double> parameters (Iterative.hxx:47-108). */
typedef struct {
  double tol;          /* SetTolerance; Seldon default 1e-6 */
  int max_iter;        /* SetMaxNumberIteration; default 100 */
  int restart;         /* SetRestart (GMRES m); default 10 */
  int print_level;     /* 0 silent, 1 every 100 iterations, 6 every iteration */
  int init_guess_null; /* SetInitGuess: 1 -> x is zeroed, 0 -> x is used */
} sb2_iter_params;

/* What the solve reports back. */
typedef struct {
  int nb_iter;          /* Iteration::GetNumberIteration() at exit */
  int error_code;       /* Iteration::ErrorCode(): 0, -2 (max_iter), or the
                           driver's breakdown code (1 to 5) */
  int init_failed;      /* 1 when Init() found a zero right-hand side (for
                           TfQmr a zero preconditioned initial residual) */
  int hist_len;         /* entries written to the caller's history buffer */
  double facteur_reste; /* 1/||r_init|| (Iteration::GetFactor) */
  double last_residual; /* relative residual of the last Finished() test */
} sb2_iter_result;

/* Seldon's drivers.  M == NULL means the identity (Preconditioner_Base).
 * hist/hist_it (host, may be NULL) receive, for every Finished() test, the
 * relative residual and the iteration number it was tested at (hist_cap
 * entries at most) -- the lines Seldon prints at print_level 6.
 * Cg.cxx:45-116, BiCgStab.cxx:43-145, Gmres.cxx:44-183. */
int sb2_cg(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
           const sb2_iter_params* params, sb2_iter_result* result, double* hist,
           int* hist_it, int hist_cap, void* stream);
int sb2_bicgstab(const sb2_csr* A, const sb2_precond* M, double* x,
                 const double* b, const sb2_iter_params* params,
                 sb2_iter_result* result, double* hist, int* hist_it,
                 int hist_cap, void* stream);
int sb2_gmres(const sb2_csr* A, const sb2_precond* M, double* x,
              const double* b, const sb2_iter_params* params,
              sb2_iter_result* result, double* hist, int* hist_it,
              int hist_cap, void* stream);

/* Seldon's Cgs (Cgs.cxx:45-132) and TfQmr (TfQmr.cxx:44-243), with the
 * arguments, history and error codes of sb2_cg.  Cgs preconditions on the
 * right and tests the true residual ||b - A x|| / ||b|| twice per loop
 * (nb_iter advances by 2, codes 1 and 2 for its two breakdowns).  TfQmr
 * preconditions on the left and tests the quasi-residual bound
 * tau sqrt(m + 1) / ||r0|| with r0 = M^{-1}(b - A x0) after each half step
 * (codes 1 to 5); a zero r0 returns at once as a zero right-hand side does.
 * The identity and Jacobi run as one persistent kernel per solve; SOR and
 * ILUT drive the same device operations from the host, one at a time. */
int sb2_cgs(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
            const sb2_iter_params* params, sb2_iter_result* result, double* hist,
            int* hist_it, int hist_cap, void* stream);
int sb2_tfqmr(const sb2_csr* A, const sb2_precond* M, double* x,
              const double* b, const sb2_iter_params* params,
              sb2_iter_result* result, double* hist, int* hist_it,
              int hist_cap, void* stream);

/* Seldon's MinRes (MinRes.cxx:46-153) for symmetric, possibly indefinite,
 * systems with a symmetric preconditioner; arguments, history and error
 * codes of sb2_cg (codes 1 and 2 for its two breakdowns).  The stopping
 * test is on the recurrence's residual estimate, ||b|| times the product
 * of the Givens sines so far.  The identity and Jacobi run as one
 * persistent kernel per solve; SOR and ILUT drive the device operations
 * from the host, one at a time. */
int sb2_minres(const sb2_csr* A, const sb2_precond* M, double* x,
               const double* b, const sb2_iter_params* params,
               sb2_iter_result* result, double* hist, int* hist_it,
               int hist_cap, void* stream);

/* Seldon's Gcr (Gcr.cxx:45-141): restarted generalized conjugate residuals,
 * left preconditioned, restart m = params->restart; arguments, history and
 * error codes of sb2_cg (code 1 for its breakdown; like the reference, a
 * breakdown ends only the current cycle).  Every cycle logs the outer and
 * the inner Finished() test, as the reference's two Iteration objects do.
 * Where the reference never returns -- a cycle that takes no step (a
 * breakdown at its first product, or m = 0), which every later cycle then
 * repeats -- the solve stops after that cycle.  The identity and Jacobi
 * with m <= 16 run as one persistent kernel per solve; larger restarts, SOR
 * and ILUT drive the device operations from the host. */
int sb2_gcr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
            const sb2_iter_params* params, sb2_iter_result* result, double* hist,
            int* hist_it, int hist_cap, void* stream);

/* Seldon's BiCgStabl (BiCgStabl.cxx:43-180): BiCGSTAB(l) with l =
 * params->restart >= 1 (l = 0 gives SB2_ERR_INVALID_VALUE: the reference
 * reads past its gamma vector there), right preconditioning (x is mapped
 * back by M^{-1} at the end, as the reference does); arguments, history and
 * error codes of sb2_cg (codes 1 and 2; like the reference, a breakdown
 * ends only the BiCG part of the cycle).  Where the reference can repeat a
 * cycle for ever (one that counts no iteration) the solve stops after it.
 * The identity and Jacobi with l <= 16 run as one persistent kernel per
 * solve; larger l, SOR and ILUT drive the device operations from the
 * host. */
int sb2_bicgstabl(const sb2_csr* A, const sb2_precond* M, double* x,
                  const double* b, const sb2_iter_params* params,
                  sb2_iter_result* result, double* hist, int* hist_it,
                  int hist_cap, void* stream);

/* Seldon's QCgs (QCgs.cxx:46-165): Cgs with a quasi-minimal smoothing
 * step, right preconditioning; arguments, history and error codes of
 * sb2_cg (codes 1 to 3).  The test is on the smoothed residual, and x is
 * replaced by M^{-1} x_qcgs at the end, breakdown or not, as in the
 * reference.  The identity and Jacobi run as one persistent kernel per
 * solve; SOR and ILUT drive the device operations from the host. */
int sb2_qcgs(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream);

/* Seldon's BiCg (BiCg.cxx:46-134): biconjugate gradients with one product
 * by A and one by A^T per loop (for a general matrix the transpose is built
 * once per handle, as for sb2_spmv with trans; symmetric storage is its own
 * transpose) and M^{-1}, M^{-T} on the two residuals; arguments, history and
 * error codes of sb2_cg (codes 1 and 2).  The identity and Jacobi run as
 * one persistent kernel per solve; SOR and ILUT drive the device
 * operations from the host. */
int sb2_bicg(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream);

/* Seldon's CoCg (CoCg.cxx:45-116), conjugate orthogonal CG for complex
 * symmetric systems.  In real arithmetic its steps are Cg's, so it runs
 * sb2_cg's engines and returns sb2_cg's results (the reference's CoCg and
 * Cg agree bit for bit as well). */
int sb2_cocg(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream);

/* Seldon's Cgne (Cgne.cxx:40-127): CG on the normal equations
 * A^T A x = A^T b, with M^{-T} then M^{-1} applied to the residual;
 * arguments, history and error codes of sb2_cg (codes 1 and 2).  The test
 * is on ||r|| / ||A^T b||, the first one on ||A^T b|| even from an initial
 * guess, and the count advances by two per loop, as in the reference.  The
 * identity and Jacobi run as one persistent kernel per solve; SOR and ILUT
 * drive the device operations from the host. */
int sb2_cgne(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream);

/* Seldon's BiCgcr (BiCgcr.cxx:44-118): biconjugate conjugate residuals, one
 * product a step; arguments, history and error codes of sb2_cg (codes 1 and
 * 2).  The count starts at 1, as in the reference, which counts the first
 * product before its first test; the test is on the unpreconditioned
 * residual.  The identity and Jacobi run as one persistent kernel per
 * solve; SOR and ILUT drive the device operations from the host. */
int sb2_bicgcr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream);

/* Seldon's Lsqr (Lsqr.cxx:40-135): Golub-Kahan bidiagonalisation with the
 * products by A and A^T; arguments, history and error codes of sb2_cg
 * (codes 1 to 3).  The preconditioner is not used (any valid handle, or
 * NULL).  As in the reference, an initial guess enters only the first test
 * (on ||b - A x0|| / ||b||): x is zeroed and the iteration starts from b.
 * The later tests are on |phi_bar| / ||b|| and the count advances by two a
 * step.  One persistent kernel per solve. */
int sb2_lsqr(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
             const sb2_iter_params* params, sb2_iter_result* result, double* hist,
             int* hist_it, int hist_cap, void* stream);

/* Seldon's QmrSym (QmrSym.cxx:41-165): QMR for symmetric systems, one
 * product a step; arguments and history of sb2_cg.  Error codes are the
 * reference's Fail codes 1, 3, 4, 5 and 6 (its messages number them #1 to
 * #5).  The identity and Jacobi run as one persistent kernel per solve; SOR
 * and ILUT drive the device operations from the host. */
int sb2_qmrsym(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream);

/* Seldon's Symmlq (Symmlq.cxx:45-161): Lanczos with an LQ factorisation, one
 * product a step; arguments and history of sb2_cg, no breakdown code.  The
 * first test is on ||b|| even from an initial guess, the later ones on the
 * recurrence's estimate; x takes its last correction after the loop however
 * it ended, as in the reference.  The identity and Jacobi run as one
 * persistent kernel per solve; SOR and ILUT drive the device operations
 * from the host. */
int sb2_symmlq(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
               const sb2_iter_params* params, sb2_iter_result* result, double* hist,
               int* hist_it, int hist_cap, void* stream);

/* Gmres(m) with classical Gram-Schmidt applied twice (CGS2) in place of the
 * reference's modified Gram-Schmidt loop (Gmres.cxx:127-132): each Arnoldi
 * step projects the new vector on the whole basis at once, twice, so it
 * takes three grid-wide reductions where the modified order takes i + 2.
 * Restarts, Givens rotations, back-solve, stopping rule, error codes and
 * history are those of sb2_gmres (Gmres.cxx:44-183); the iterates agree with
 * the reference's to rounding, not bit for bit.  M: NULL (identity) or
 * Jacobi; restart (m) <= 32.  Other preconditioners or a larger restart give
 * SB2_ERR_NOT_SUPPORTED.  No counterpart in the reference (a labelled
 * variant of its Gmres). */
int sb2_gmres_cgs2(const sb2_csr* A, const sb2_precond* M, double* x,
                   const double* b, const sb2_iter_params* params,
                   sb2_iter_result* result, double* hist, int* hist_it,
                   int hist_cap, void* stream);

/* Cg with the identity preconditioner that allocates no memory at all.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- code whose device memory is entirely owned by another
 * allocator (a framework that reserves the whole GPU up front), latency-bound
 * loops that must not pay cudaMalloc's implicit device synchronization, and
 * plugin hosts that forbid libraries to allocate.  Such a caller creates the
 * matrix beforehand and passes x and b (device memory it owns).
 * The work vectors live in a fixed array inside this library, sized for
 * n <= 131072 rows (about 3.3 MB, held on every GPU that loads the library
 * until the process exits); larger systems are rejected with
 * SB2_ERR_INVALID_VALUE.  The first call on a device looks up that array's
 * device address, which is kept for the life of the process:
 * cudaDeviceReset destroys the array with the context, and this entry point
 * must not be called on that device afterwards (matrix handles made before
 * the reset are gone too).  All
 * calls on a device share the one array: calls that overlap on the GPU
 * (other streams, other host threads) race and must be serialized by the
 * caller.  The call returns after the solve has finished: it reads the
 * result record back to the host.  Iteration count, error code and last
 * residual are reported; no residual history.
 * It runs the persistent CG kernel of sb2_cg (M == NULL).  sb2_cg runs that
 * same kernel, and gives the same bits, when the system is below the chained
 * size (sb2_krylov_set_config) and its cluster-resident form is off
 * (sb2_krylov_set_cluster(0)); with the cluster form on, sb2_cg groups its
 * sums by cluster rank and agrees to rounding only. */
int sb2_cg_noalloc(const sb2_csr* A, double* x, const double* b,
                   const sb2_iter_params* params, sb2_iter_result* result, void* stream);

/* ------------------------------------------------------------ mixed precision */

/* Iterative refinement with FP32 inner Krylov solves (FP32 values, vectors
 * and accumulation) inside an FP64 outer loop: the residual r = b - A x, the
 * solution update and the stopping test stay in FP64.  New form beside the
 * reference's drivers (no counterpart in Seldon); the inner solvers follow
 * Cg.cxx:45-116 and Gmres.cxx:44-183, the stopping rule Iterative.cxx:272-319.
 *
 * solver 1 (GMRES) is restarted GMRES(restart) whose restarts are the
 * refinement steps: each cycle builds its Krylov basis in FP32 (FP32 products,
 * basis vectors and per-thread sums, orthogonalized by CGS2), while the
 * Hessenberg matrix, its Givens rotations and back-solve, the update
 * x += V y and the residual that starts the next cycle are FP64.  A cycle
 * ends after `restart` steps, when its residual estimate has dropped by
 * inner_tol, or when the estimate of ||M^-1 r|| / ||M^-1 r0|| is below tol;
 * the solve stops when the FP64 ||b - A x|| / ||b|| < tol at a restart.
 * max_inner bounds the Arnoldi steps, max_outer the cycles; mode is not
 * read. */
typedef struct {
  double tol;          /* outer target: ||b - A x|| / ||b|| < tol (FP64) */
  double inner_tol;    /* relative residual reduction of each inner solve */
  int max_outer;       /* refinement steps at most */
  int max_inner;       /* iterations of one inner solve at most */
  int solver;          /* inner solver: 0 = CG, 1 = GMRES */
  int restart;         /* GMRES: steps per cycle (<= 32; <= 0 means 30) */
  int init_guess_null; /* 1: x = 0; 0: start from x */
  int mode;            /* 0: reliable updates -- one FP32 CG run whose residual
                          is replaced by the FP64 true residual each time it has
                          dropped by inner_tol (the search direction carries
                          on, so the iteration count stays near FP64 CG's);
                          1: restarted refinement -- a fresh FP32 CG solve of
                          A d = r to inner_tol per outer step */
} sb2_ir_params;

typedef struct {
  int outer_iter;      /* FP64 corrections applied */
  int inner_iter;      /* FP32 iterations in all */
  int error_code;      /* 0 converged, -2 stopped at max_outer */
  int init_failed;     /* zero right-hand side (x untouched) */
  int hist_len;        /* entries written to hist */
  double rel_residual; /* final FP64 ||b - A x|| / ||b|| */
} sb2_ir_result;

/* M: NULL (identity) or a Jacobi preconditioner of A (applied in FP32 inside
 * the inner solves, in FP64 to the outer residual).  hist (host, may be NULL)
 * receives the FP64 relative residual before each refinement step and at
 * the end. */
int sb2_ir_solve(const sb2_csr* A, const sb2_precond* M, double* x, const double* b,
                 const sb2_ir_params* params, sb2_ir_result* result, double* hist,
                 int hist_cap, void* stream);

/* ------------------------------------------------------------ differentiation */
/* Pieces of the hand-written adjoint of x = A^{-1} b for a loss L(x): solve
 * A^T lambda = dL/dx with sb2_cg (symmetric A) or sb2_bicgstab / sb2_gmres
 * (general A: pass the transpose), then dL/db = lambda and the kernels below.
 * No counterpart in the reference (new form beside its drivers). */

/* New values on the same pattern (general RowSparse matrices only): val[nnz]
 * in the stored order, on the device (on_device = 1) or the host.  Derived
 * copies (diagonal, FP32 values, transpose) are rebuilt on their next use. */
int sb2_csr_set_values(sb2_csr* A, const double* val, int on_device, void* stream);

/* grad_val[k] = alpha * lambda[row(k)] * x[ind[k]] for every stored entry k:
 * with alpha = -1, dL/dA_ij restricted to the pattern. */
int sb2_grad_pattern(const sb2_csr* A, double alpha, const double* lambda, const double* x,
                     double* grad_val, void* stream);

/* grad[e] = -(lambda[i] - lambda[j]) * (x[i] - x[j]) for edges e = (ei[e], ej[e]):
 * dL/dtheta_e of a weighted graph Laplacian (A_ii, A_jj += theta_e,
 * A_ij = A_ji -= theta_e).  ei, ej, lambda, x and grad are device arrays;
 * the call takes no vertex count, so every ei[e] and ej[e] must already lie
 * in [0, length of lambda and x): the indices are not checked (the Python
 * autograd wrapper builds them from the graph it was given). */
int sb2_grad_edges(int nedges, const int* ei, const int* ej, const double* lambda,
                   const double* x, double* grad, void* stream);

/* ------------------------------------------------------------ batched solves */

/* A batch of independent square systems, held as one block-diagonal CSR
 * operator: system s owns rows [sys_row[s], sys_row[s+1]) and its entries may
 * only reference columns in that range (checked).  New form beside the
 * reference's drivers (no counterpart in Seldon): each system is solved as
 * Cg.cxx:45-116 would, with the Iterative.cxx:272-319 stopping rule. */
typedef struct sb2_batch sb2_batch;

typedef struct {
  double tol;          /* per system: stop when ||b - A x|| / ||b|| < tol (FP64) */
  double update_ratio; /* mode 0: FP64 correction when the FP32 residual has
                          dropped by this factor (e.g. 1e-2) */
  int max_iter;        /* iterations per system at most */
  int mode;            /* 0: FP32 CG with FP64 reliable updates; 1: FP64 CG */
  int init_guess_null; /* 1: x = 0; 0: start from x */
} sb2_batch_params;

typedef struct {
  int converged;           /* systems that met tol */
  int max_iter;            /* largest iteration count of a system */
  long long total_iter;    /* iterations summed over the systems */
  double max_rel_residual; /* worst final FP64 relative residual */
} sb2_batch_result;

/* HOST arrays: sys_row[nsys+1], ptr[m+1], ind[nnz] (global columns), val[nnz]. */
int sb2_batch_create(int nsys, const int* sys_row, const int* ptr, const int* ind,
                     const double* val, sb2_batch** out);
int sb2_batch_destroy(sb2_batch* B);

/* Solve every system in ONE persistent launch (CTAs take systems from a
 * queue, largest first).  x, b: device vectors of all rows.  d_iters /
 * d_relres (device, may be NULL): per-system iteration count and final
 * relative residual.  With result == NULL the call only enqueues work on
 * `stream` (no host synchronization, so it can be captured in a CUDA graph);
 * with result != NULL it waits and summarizes (d_iters and d_relres needed). */
int sb2_batch_solve(const sb2_batch* B, double* x, const double* b,
                    const sb2_batch_params* params, int* d_iters, double* d_relres,
                    sb2_batch_result* result, void* stream);

/* The solve's plan, chosen per size class of the systems:
 *   threads   CTA size (128, 256 or 512) of the systems a whole CTA solves
 *   warp_max  systems of at most this many rows are solved by one warp each
 *             (a CTA holds several of them), with shuffle reductions and no
 *             CTA barrier; 0: every system gets a CTA
 * The queue hands systems out largest first, so a CTA that takes a system of
 * at most warp_max rows turns to warps for the rest of the launch.
 * Autotuner: times the solve of this batch (x is overwritten) under each
 * candidate plan (threads 128, 256, 512 by warp_max 0, 256, 1024) and keeps
 * the fastest for later solves.  The choice is cached per (histogram of the
 * systems' sizes in power-of-two classes, mode): a later batch with the same
 * histogram takes it without timing. */
int sb2_batch_autotune(sb2_batch* B, double* x, const double* b,
                       const sb2_batch_params* params, void* stream);
int sb2_batch_set_threads(sb2_batch* B, int threads);
int sb2_batch_get_threads(const sb2_batch* B);
int sb2_batch_set_plan(sb2_batch* B, int threads, int warp_max);
int sb2_batch_get_plan(const sb2_batch* B, int* threads, int* warp_max);

/* Cluster part of the plan, for batches with fewer large systems than the
 * GPU has CTA slots: the launch groups its CTAs in thread-block clusters of
 * `cluster` CTAs (2, 4, 8 or 16; 0: none), and the systems of more than
 * cluster_min rows are each solved by a whole cluster (rows spread over its
 * CTAs, reductions through distributed shared memory and the cluster's
 * barrier).  The smaller systems then go to single CTAs and warps as the
 * rest of the plan says.  sb2_batch_set_plan clears it; the autotuner also
 * times clusters of 4 and 16 CTAs for the systems above half or an eighth of
 * the largest, and caches the cluster part with the rest.  A cluster plan
 * that the GPU cannot schedule makes sb2_batch_solve return
 * SB2_ERR_NOT_SUPPORTED. */
int sb2_batch_set_cluster_plan(sb2_batch* B, int cluster, int cluster_min);
int sb2_batch_get_cluster_plan(const sb2_batch* B, int* cluster, int* cluster_min);

/* Size from which Cg (identity or Jacobi) runs as a chain of full-occupancy
 * kernels (one per pass, scalars in device memory) instead of one
 * persistent kernel; BiCgStab does from three times that size.  The
 * default, 3500000 rows, is where Cg's two forms cross on 7-point Poisson
 * matrices on a B200; BiCgStab's persistent kernel is still the faster at
 * 7.1M rows.  The forms group their reductions differently, so their
 * iterates agree to rounding.  0 runs both drivers chained at every size.
 * Returns the previous value.  No counterpart in the reference (a tuning
 * knob of this engine). */
int sb2_krylov_set_config(int chain_min_n);

/* Cluster-resident CG (on by default): a system whose matrix and vectors fit
 * the shared memory of one thread-block cluster (up to 16 CTAs on 16 SMs)
 * runs Cg inside that cluster, exchanging data through distributed shared
 * memory and synchronizing with hardware cluster barriers; the arithmetic is
 * the same as the persistent kernel's.  0 turns it off (the persistent
 * kernel runs instead); 1 turns it on with up to 16 CTAs; 2, 4, 8 or 16 turn
 * it on with at most that many.  Returns the previous setting (0 or the
 * cap).  No counterpart in the reference (a tuning knob of this engine). */
int sb2_krylov_set_cluster(int on);

/* Cg, BiCgStab and Gmres with an SOR or ILUT preconditioner: 1 (default)
 * runs them as chains of device kernels whose scalars (rho, alpha, beta,
 * omega, Gmres's Hessenberg matrix, rotations and s, the residual and the
 * stop flags) stay in device memory, the preconditioner's sweeps enqueued
 * between them, with no host synchronization per iteration (Gmres: the host
 * reads the state once per chunk of Arnoldi steps, to place the end of each
 * cycle); 0 runs the host-driven loop of library calls (a dot product
 * returned to the host each time, as the reference's generic driver does).
 * The two group their reductions differently, so their iterates agree to
 * rounding.  Returns the previous setting.  No counterpart in the reference
 * (a tuning knob of this engine). */
int sb2_krylov_set_pcg(int device_resident);

/* Device-side wait limit for the fused solvers' grid barriers, in
 * milliseconds (default 2000).  Values <= 0 leave it unchanged.  Returns the
 * previous value (rounded up to whole milliseconds).  No counterpart in the
 * reference (the reference runs on the host and never waits on a device). */
int sb2_set_wait_limit_ms(int ms);

/* The same limit in microseconds (>= 1; values <= 0 leave it unchanged);
 * returns the previous value in microseconds.  A limit below the time one
 * CTA may wait for the slowest at a grid barrier makes the fused solvers end
 * with SB2_ERR_TIMEOUT: every CTA leaves the kernel, the context stays
 * usable, and the next call with a longer limit solves normally.  The TMA
 * product's ring waits keep a floor of 1 s whatever this limit is.  No
 * counterpart in the reference. */
int sb2_set_wait_limit_us(int us);

#ifdef __cplusplus
}
#endif
#endif /* SELDON_B200_H */
