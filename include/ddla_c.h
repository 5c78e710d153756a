/*
 * ddla_c.h -- C ABI of the B200 Cholesky-path library (libddla_c.so).
 *
 * This is the drop-in boundary: the same exported names, argument order and
 * status convention as the reference's generated C ABI
 * (fortran/ddla_c_api.cpp), which python/ddla/_c_api.py binds with ctypes.
 * Each declaration cites the reference export it replaces.
 *
 * Conventions (ddla_c_api.cpp:1-27, 44-52): every call returns an int status
 * 0 success, 1 invalid handle, 2 invalid value, 3 alloc failed,
 * 4 backend unavailable, 5 internal (device) error, 6 a C++ exception escaped
 * (its text via ddla_c_error_string(6), kept per thread).  The handle travels
 * as void*; matrices are device pointers of a GPU handle; descriptors are the
 * ScaLAPACK int[9] arrays; info is a host int* except for ddla_?_potrf, whose
 * info is a device int* (asynchronous, like the reference's GPU potrf).
 * Only the 1x1 process grid is served and only the GPU backend exists.
 */
#ifndef DDLA_C_H
#define DDLA_C_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- lifecycle, grid and memory -------------------------------------- */
const char* ddla_c_error_string(int status);                                  /* ddla_c_api.cpp:91 */
int ddla_c_init_backend(void** handle, int backend);                          /* ddla_c_api.cpp:100 */
int ddla_c_set(void* handle, int f_comm, int nprows, int npcols, char major); /* ddla_c_api.cpp:115 */
int ddla_c_set_communication(void* handle, int communication);                /* ddla_c_api.cpp:134 */
/* Process grids of more than one rank (the reference forms them from an MPI
 * communicator, ddla_c_api.cpp:115 / src/ddla_handle_t.cpp:94-201; MPI is not
 * part of this build).  A local group joins ranks that are threads of this
 * process, one handle per rank; NCCL joins ranks that are processes (rank 0
 * makes the 128-byte clique id, every rank passes it).  Additive entry points. */
int ddla_c_local_group_create(void** group, int nranks, double timeout_s);
int ddla_c_local_group_destroy(void* group);
int ddla_c_set_local_group(void* handle, void* group, int rank, int nprows, int npcols, char major);
int ddla_c_nccl_available(void);
int ddla_c_nccl_unique_id(void* id128);
int ddla_c_set_nccl(void* handle, const void* id128, int nranks, int rank, int nprows, int npcols, char major);
int ddla_c_get_communication(void* handle, int* communication);               /* ddla_c_api.cpp:144 */
int ddla_c_communication_available(void* handle, int communication);          /* ddla_c_api.cpp:156 */
int ddla_c_destroy(void** handle);                                            /* ddla_c_api.cpp:165 */
int ddla_c_backend_available(int backend);                                    /* ddla_c_api.cpp:178 */
int ddla_c_get_backend(void* handle);                                         /* ddla_c_api.cpp:184 */
int ddla_c_grid_dims(void* handle, int* nprows, int* npcols);                 /* ddla_c_api.cpp:190 */
int ddla_c_grid_coords(void* handle, int* myprow, int* mypcol);               /* ddla_c_api.cpp:197 */
int ddla_c_rank(void* handle);                                                /* ddla_c_api.cpp:204 */
int ddla_c_size(void* handle);                                                /* ddla_c_api.cpp:210 */
int ddla_c_descinit(int* desc, void* handle, int m, int n, int mb, int nb, int irsrc, int icsrc,
                    int lld);                                                 /* ddla_c_api.cpp:216 */
int ddla_c_numloc(int n, int nb, int iproc, int srcproc, int nprocs);         /* ddla_c_api.cpp:224 */
int ddla_c_malloc(void* handle, void** ptr, long long bytes);                 /* ddla_c_api.cpp:229 */
int ddla_c_free(void* handle, void* ptr);                                     /* ddla_c_api.cpp:236 */
int ddla_c_memcpy(void* handle, void* dst, const void* src, long long bytes); /* ddla_c_api.cpp:242 */
int ddla_c_memcpy2d(void* handle, void* dst, long long dpitch, const void* src, long long spitch, long long width,
                    long long height);                                        /* ddla_c_api.cpp:249 */
int ddla_c_memset(void* handle, void* ptr, int value, long long bytes);       /* ddla_c_api.cpp:260 */
int ddla_c_synchronize(void* handle);                                         /* ddla_c_api.cpp:267 */
int ddla_c_default_comm(void);                                                /* ddla_c_api.cpp:304 */
int ddla_c_comm_rank(int f_comm);                                             /* ddla_c_api.cpp:310 */
int ddla_c_comm_size(int f_comm);                                             /* ddla_c_api.cpp:319 */
void ddla_c_finalize(void);                                                   /* ddla_c_api.cpp:328 */
int ddla_c_bcast_dims(int f_comm, int* m, int* n, int* type_char, int root);  /* ddla_c_api.cpp:339 */

/* ---- 1x1-grid gather / scatter (host global <-> device local) ---------- */
int ddla_s_gather(void* h, int m, int n, const void* A, int ia, int ja, const int* descA, int root, void* dst,
                  int lddst); /* ddla_c_api.cpp:515 (ddla_c_gather and its s/d/z siblings) */
int ddla_d_gather(void* h, int m, int n, const void* A, int ia, int ja, const int* descA, int root, void* dst,
                  int lddst);
int ddla_c_gather(void* h, int m, int n, const void* A, int ia, int ja, const int* descA, int root, void* dst,
                  int lddst);
int ddla_z_gather(void* h, int m, int n, const void* A, int ia, int ja, const int* descA, int root, void* dst,
                  int lddst);
int ddla_s_scatter(void* h, int m, int n, void* A, int ia, int ja, const int* descA, int root, const void* src,
                   int ldsrc); /* ddla_c_api.cpp:551 (ddla_c_scatter and its s/d/z siblings) */
int ddla_d_scatter(void* h, int m, int n, void* A, int ia, int ja, const int* descA, int root, const void* src,
                   int ldsrc);
int ddla_c_scatter(void* h, int m, int n, void* A, int ia, int ja, const int* descA, int root, const void* src,
                   int ldsrc);
int ddla_z_scatter(void* h, int m, int n, void* A, int ia, int ja, const int* descA, int root, const void* src,
                   int ldsrc);

/* ---- the Cholesky path ------------------------------------------------- */
/* ddla_c_api.cpp:1155-1189 */
int ddla_s_ppotrf(void* handle, char uplo, int n, void* A, int ia, int ja, const int* descA, int* info);
int ddla_d_ppotrf(void* handle, char uplo, int n, void* A, int ia, int ja, const int* descA, int* info);
int ddla_c_ppotrf(void* handle, char uplo, int n, void* A, int ia, int ja, const int* descA, int* info);
int ddla_z_ppotrf(void* handle, char uplo, int n, void* A, int ia, int ja, const int* descA, int* info);
/* ddla_c_api.cpp:1263-1297 */
int ddla_s_ppotrs(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A, const int* descA,
                  void* B, const int* descB);
int ddla_d_ppotrs(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A, const int* descA,
                  void* B, const int* descB);
int ddla_c_ppotrs(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A, const int* descA,
                  void* B, const int* descB);
int ddla_z_ppotrs(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A, const int* descA,
                  void* B, const int* descB);
/* ddla_c_api.cpp:1299-1333 */
int ddla_s_pposv(void* handle, char side, char uplo, char trans, int n, int nrhs, void* A, int ia, int ja,
                 const int* descA, void* B, int ib, int jb, const int* descB, int* info);
int ddla_d_pposv(void* handle, char side, char uplo, char trans, int n, int nrhs, void* A, int ia, int ja,
                 const int* descA, void* B, int ib, int jb, const int* descB, int* info);
int ddla_c_pposv(void* handle, char side, char uplo, char trans, int n, int nrhs, void* A, int ia, int ja,
                 const int* descA, void* B, int ib, int jb, const int* descB, int* info);
int ddla_z_pposv(void* handle, char side, char uplo, char trans, int n, int nrhs, void* A, int ia, int ja,
                 const int* descA, void* B, int ib, int jb, const int* descB, int* info);
/* ddla_c_api.cpp:2150-2180 (info is a DEVICE int*) */
int ddla_s_potrf(void* handle, char uplo, int n, void* A, int lda, void* info);
int ddla_d_potrf(void* handle, char uplo, int n, void* A, int lda, void* info);
int ddla_c_potrf(void* handle, char uplo, int n, void* A, int lda, void* info);
int ddla_z_potrf(void* handle, char uplo, int n, void* A, int lda, void* info);

/* ddla_c_api.cpp:1191-1225: bottom-right Cholesky, A = U*U^H ('U') or L^H*L ('L');
 * info (host int*) is 0 or the failed pivot's index */
int ddla_s_potrf_bottom_right(void* handle, char uplo, int n, void* A, int lda, int* info);
int ddla_d_potrf_bottom_right(void* handle, char uplo, int n, void* A, int lda, int* info);
int ddla_c_potrf_bottom_right(void* handle, char uplo, int n, void* A, int lda, int* info);
int ddla_z_potrf_bottom_right(void* handle, char uplo, int n, void* A, int lda, int* info);
/* ddla_c_api.cpp:1227-1261: the same through an int[9] descriptor (1x1 grid) */
int ddla_s_ppotrf_bottom_right(void* handle, char uplo, int n, void* A, const int* descA, int* info);
int ddla_d_ppotrf_bottom_right(void* handle, char uplo, int n, void* A, const int* descA, int* info);
int ddla_c_ppotrf_bottom_right(void* handle, char uplo, int n, void* A, const int* descA, int* info);
int ddla_z_ppotrf_bottom_right(void* handle, char uplo, int n, void* A, const int* descA, int* info);

/* diag_logdet has no C export in the reference (its C++ template is
 * include/ddla/ddla.h:2900-2902); these add one.  result receives two reals
 * of the matrix's real type: log magnitude, phase in (-pi, pi]. */
int ddla_s_diag_logdet(void* handle, int n, const void* A, int lda, void* result);
int ddla_d_diag_logdet(void* handle, int n, const void* A, int lda, void* result);
int ddla_c_diag_logdet(void* handle, int n, const void* A, int lda, void* result);
int ddla_z_diag_logdet(void* handle, int n, const void* A, int lda, void* result);
/* pdiag_logdet (reference include/ddla/ddla.h:2914-2915, no C export there):
 * the same through an int[9] descriptor, leading dimension LLD_ */
int ddla_s_pdiag_logdet(void* handle, int n, const void* A, const int* descA, void* result);
int ddla_d_pdiag_logdet(void* handle, int n, const void* A, const int* descA, void* result);
int ddla_c_pdiag_logdet(void* handle, int n, const void* A, const int* descA, void* result);
int ddla_z_pdiag_logdet(void* handle, int n, const void* A, const int* descA, void* result);
/* pdiag_logdet on a pr x pc grid, split at the reference's one exchange step
 * (src/PBLAS/pdiag_logdet.cpp:41-47, MPI_Allreduce of four doubles; no C export
 * there): ddla_?_pdiag_logdet_local writes this rank's state[5] = {magnitude,
 * phase, zero, negative parity, nonfinite} over the diagonal entries its local
 * matrix holds (descA checked against the pr x pc grid, rank (row, col)); the
 * caller sums the five doubles over all ranks; ddla_c_pdiag_logdet_finish turns
 * the sums into the log-determinant (result: two floats if single, else two
 * doubles), status 6 "nonfinite diagonal" on every rank if any rank saw one. */
int ddla_s_pdiag_logdet_local(void* handle, int n, const void* A, const int* descA, int pr, int pc, int row, int col,
                              double* state);
int ddla_d_pdiag_logdet_local(void* handle, int n, const void* A, const int* descA, int pr, int pc, int row, int col,
                              double* state);
int ddla_c_pdiag_logdet_local(void* handle, int n, const void* A, const int* descA, int pr, int pc, int row, int col,
                              double* state);
int ddla_z_pdiag_logdet_local(void* handle, int n, const void* A, const int* descA, int pr, int pc, int row, int col,
                              double* state);
int ddla_c_pdiag_logdet_finish(const double* total, int single, void* result);
/* phegst (reference include/ddla/ddla.h:2560-2562, no C export there): the
 * type-1 Hermitian-definite reduction of A with the factor held in F */
int ddla_s_phegst(void* handle, char uplo, int n, void* A, const int* descA, const void* F, const int* descF);
int ddla_d_phegst(void* handle, char uplo, int n, void* A, const int* descA, const void* F, const int* descF);
int ddla_c_phegst(void* handle, char uplo, int n, void* A, const int* descA, const void* F, const int* descF);
int ddla_z_phegst(void* handle, char uplo, int n, void* A, const int* descA, const void* F, const int* descF);
/* The mixed gemmVbatched overloads (reference include/ddla/ddla.h:1878-1939, C++
 * only there): _rc takes a real A and a complex B, _cr a complex A and a real B;
 * alpha, beta and C are complex (the c / z prefix is their type). */
int ddla_c_gemm_vbatched_rc(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                            const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                            void** d_C, int* d_ldc, int batch_count);
int ddla_c_gemm_vbatched_cr(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                            const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                            void** d_C, int* d_ldc, int batch_count);
int ddla_z_gemm_vbatched_rc(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                            const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                            void** d_C, int* d_ldc, int batch_count);
int ddla_z_gemm_vbatched_cr(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                            const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                            void** d_C, int* d_ldc, int batch_count);
/* gemmVbatched (reference include/ddla/ddla.h:1836-1849, a C++ template with
 * no C export there): the batched GEMM over device-resident size, leading-
 * dimension and pointer arrays; alpha and beta point to one host scalar of the
 * routine's type.  Errors as the template's (ST_EXCEPTION with its message). */
int ddla_s_gemm_vbatched(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                         const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                         void** d_C, int* d_ldc, int batch_count);
int ddla_d_gemm_vbatched(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                         const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                         void** d_C, int* d_ldc, int batch_count);
int ddla_c_gemm_vbatched(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                         const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                         void** d_C, int* d_ldc, int batch_count);
int ddla_z_gemm_vbatched(void* handle, char transA, char transB, int* d_m, int* d_n, int* d_k, const void* alpha,
                         const void* const* d_A, int* d_lda, const void* const* d_B, int* d_ldb, const void* beta,
                         void** d_C, int* d_ldc, int batch_count);
/* gemmVbatched2s (reference include/ddla/ddla.h:1851-1876, C++ only there):
 * the two-stage form; alphas and betas point to one host scalar of the
 * routine's type, c0_left is 0 or 1, segment_sizes is host memory. */
#define DDLA_GEMM_VBATCHED2S_ARGS                                                                                  \
    void *handle, char transA_0, char transB_0, int *d_m_0, int *d_n_0, int *d_k_0, const void *alpha_0,          \
        const void *const *d_A_0, int *d_lda_0, const void *const *d_B_0, int *d_ldb_0, const void *beta_0,        \
        void **d_C_0, int *d_ldc_0, char transA_1, char transB_1, int *d_m_1, int *d_n_1, int *d_k_1,             \
        const void *alpha_1, const void *const *d_AB_1, int *d_lda_1, int *d_ldb_1, const void *beta_1,            \
        void **d_C_1, int *d_ldc_1, int c0_left, int batch_count, const int *segment_sizes, int segment_count
int ddla_s_gemm_vbatched2s(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_d_gemm_vbatched2s(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_c_gemm_vbatched2s(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s(DDLA_GEMM_VBATCHED2S_ARGS);
/* The mixed gemmVbatched2s overloads (reference include/ddla/ddla.h:1893-2030,
 * C++ only there), named by the element types of (A0, B0, C0, AB1): r real,
 * z complex; C1 is complex.  alpha_0 / beta_0 point to a scalar of C0's type,
 * alpha_1 / beta_1 to a complex one.  Arguments as ddla_?_gemm_vbatched2s. */
int ddla_c_gemm_vbatched2s_rzzr(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_c_gemm_vbatched2s_zrzr(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_c_gemm_vbatched2s_rzzz(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_c_gemm_vbatched2s_zrzz(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_c_gemm_vbatched2s_zzzr(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_c_gemm_vbatched2s_rrrz(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s_rzzr(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s_zrzr(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s_rzzz(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s_zrzz(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s_zzzr(DDLA_GEMM_VBATCHED2S_ARGS);
int ddla_z_gemm_vbatched2s_rrrz(DDLA_GEMM_VBATCHED2S_ARGS);

/* The reference's internal check / size / run split of ppotrf and ppotrs
 * (src/Cholesky/cholesky_workspace.h:133-154, 207-222) exported so a caller can
 * own the device scratch: *_workspace_size reports bytes, *_run computes on
 * the caller's scratch without allocating. */
int ddla_s_ppotrf_workspace_size(void* handle, char uplo, int n, const int* descA, long long* bytes);
int ddla_d_ppotrf_workspace_size(void* handle, char uplo, int n, const int* descA, long long* bytes);
int ddla_c_ppotrf_workspace_size(void* handle, char uplo, int n, const int* descA, long long* bytes);
int ddla_z_ppotrf_workspace_size(void* handle, char uplo, int n, const int* descA, long long* bytes);
int ddla_s_ppotrf_run(void* handle, char uplo, int n, void* A, const int* descA, int* info, void* work, long long bytes);
int ddla_d_ppotrf_run(void* handle, char uplo, int n, void* A, const int* descA, int* info, void* work, long long bytes);
int ddla_c_ppotrf_run(void* handle, char uplo, int n, void* A, const int* descA, int* info, void* work, long long bytes);
int ddla_z_ppotrf_run(void* handle, char uplo, int n, void* A, const int* descA, int* info, void* work, long long bytes);
int ddla_s_ppotrs_workspace_size(void* handle, char side, int n, int nrhs, const int* descA, const int* descB,
                                 long long* bytes);
int ddla_d_ppotrs_workspace_size(void* handle, char side, int n, int nrhs, const int* descA, const int* descB,
                                 long long* bytes);
int ddla_c_ppotrs_workspace_size(void* handle, char side, int n, int nrhs, const int* descA, const int* descB,
                                 long long* bytes);
int ddla_z_ppotrs_workspace_size(void* handle, char side, int n, int nrhs, const int* descA, const int* descB,
                                 long long* bytes);

/* ddla_d_ppotrs without any allocation.  No counterpart in the reference: its
 * ppotrs always allocates workspace per call.  This entry serves callers that
 * must not allocate device memory once they run -- a serving loop that reserves
 * its whole memory budget up front, or code whose CUDA allocator belongs to
 * another framework -- by keeping the solve's few kilobytes of flags in a fixed
 * device array inside the library (128 KB, present on every device that loads
 * the library until the process exits).  Same arguments, checks and result as
 * ddla_d_ppotrs, limited to n <= 65536 and nrhs <= 256 (larger sizes return
 * status 6 with a message, before any device work).  The first call on a device
 * looks the array up, so make it before any stream capture; the address is
 * kept for the life of the process, so the device's context must not be reset
 * (cudaDeviceReset) between calls.  Calls that overlap on the GPU share the
 * array and race. */
int ddla_d_ppotrs_noalloc(void* handle, char side, char uplo, char trans, int n, int nrhs, const void* A,
                          const int* descA, void* B, const int* descB);

/* Mixed-precision solve (no reference counterpart; LAPACK dsposv semantics,
 * see ddla::pposv_mixed in include/ddla/ddla.h).  precision: 'B' BF16 or 'T'
 * TF32 tensor-core factor, 'D' plain FP64.  report (may be NULL) receives
 * {double iter, double gmres, double shift, double backward_error}. */
int ddla_d_pposv_mixed(void* handle, char uplo, char precision, int n, int nrhs, void* A, const int* descA,
                       const void* B, const int* descB, void* X, const int* descX, int* info, double* report);
/* The same with A, B and X in host memory (pinned for the overlap; see
 * ddla::pposv_mixed_host): A's lower part streams to the device by column
 * panels while the arrived panels are factored.  No reference counterpart. */
int ddla_d_pposv_mixed_host(void* handle, char uplo, char precision, int n, int nrhs, const void* A, int lda,
                            const void* B, int ldb, void* X, int ldx, int* info, double* report);

/* Batched uneven Cholesky factor + solve + log-determinant in one persistent
 * launch (no reference counterpart; ddla::posvVbatched, VbatchedPlan and
 * vbatchedAutotune in include/ddla/ddla_batched.h, which give the semantics).
 * Every array argument is device resident, as for the reference's
 * gemmVbatched (include/ddla/ddla.h:1828-1849).  d_B may be NULL (factor and
 * log-determinant only).  A plan captures the launch in a CUDA graph once;
 * ddla_vbatched_plan_run replays it on the handle's stream without a host
 * synchronisation.  ddla_vbatched_tuning reports the table in use: grid,
 * widths[2], variant[len] per order bucket of 16 (len >= max_n/16 rounded up
 * to the kernel's 512 or 1024) and whether it was tuned. */
int ddla_s_posv_vbatched(void* handle, char uplo, const int* d_n, float* const* d_A, const int* d_lda,
                         float* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n);
int ddla_d_posv_vbatched(void* handle, char uplo, const int* d_n, double* const* d_A, const int* d_lda,
                         double* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n);
int ddla_s_posv_vbatched_plan(void* handle, char uplo, const int* d_n, float* const* d_A, const int* d_lda,
                              float* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n,
                              void** plan);
int ddla_d_posv_vbatched_plan(void* handle, char uplo, const int* d_n, double* const* d_A, const int* d_lda,
                              double* const* d_B, double* d_logdet, int* d_info, int batch_count, int max_n,
                              void** plan);
int ddla_vbatched_plan_run(void* plan);
int ddla_vbatched_plan_info(void* plan, int* grid, double* flops);
int ddla_vbatched_plan_destroy(void* plan);
int ddla_vbatched_autotune(void* handle, char type, int max_n);
int ddla_vbatched_tuning(void* handle, char type, int max_n, int* grid, int* widths, unsigned char* variant, int len,
                         int* tuned);

/* Negative log marginal likelihood loss = 1/2 (y^T A^-1 y + log det A) and its
 * adjoint for batches of equal-order problems (no reference counterpart;
 * ddla::cholNllBatched, gpNllBatched, cholNllGradBatched, gpNllGradBatched in
 * include/ddla/ddla_batched.h give layouts and formulas).  Device arrays:
 * A/L/W/G batch x n x n column-major, y/alpha batch x n, X batch x n x d
 * row-major, theta {l, sigma_f^2, sigma^2} (theta_stride 3 per problem, 0
 * shared), logdet/quad/info batch, grad batch x 3. */
int ddla_s_chol_nll_batched(void* handle, int batch, int n, float* A, const float* y, float* alpha, double* logdet,
                            double* quad, int* info);
int ddla_d_chol_nll_batched(void* handle, int batch, int n, double* A, const double* y, double* alpha,
                            double* logdet, double* quad, int* info);
int ddla_s_gp_nll_batched(void* handle, int batch, int n, int d, const float* X, const double* theta,
                          int theta_stride, const float* y, float* A, float* alpha, double* logdet, double* quad,
                          int* info);
int ddla_d_gp_nll_batched(void* handle, int batch, int n, int d, const double* X, const double* theta,
                          int theta_stride, const double* y, double* A, double* alpha, double* logdet, double* quad,
                          int* info);
int ddla_s_chol_nll_grad_batched(void* handle, int batch, int n, const float* L, const float* alpha, float* W,
                                 float* G);
int ddla_d_chol_nll_grad_batched(void* handle, int batch, int n, const double* L, const double* alpha, double* W,
                                 double* G);
int ddla_s_gp_nll_grad_batched(void* handle, int batch, int n, int d, const float* X, const double* theta,
                               int theta_stride, const float* L, const float* alpha, float* W, double* grad);
int ddla_d_gp_nll_grad_batched(void* handle, int batch, int n, int d, const double* X, const double* theta,
                               int theta_stride, const double* L, const double* alpha, double* W, double* grad);

/* Diagnostics (no reference counterpart: the reference has no tracing).
 * ddla_c_get_stream returns the handle's CUDA stream (ddlaGetStream of
 * include/ddla/ddla_handle_t.h:337, which the reference's C ABI does not
 * export).  ddla_c_launch_count is the number of kernels this library has
 * launched in the process.  ddla_c_profile_enable / ddla_c_profile_read switch
 * per-kernel CUDA-event timing on and read it back per kernel kind (see
 * ddlak_profile_read in ddla_kernels.h). */
int ddla_c_get_stream(void* handle, void** stream);
long long ddla_c_launch_count(void);

/* Testing aids for the failure paths (no reference counterpart in the C ABI;
 * the reference injects allocation failures with an LD_PRELOAD shim,
 * tests/pblas_alloc_failure.cpp, which cannot reach this library because it
 * links the CUDA runtime statically).  ddla_c_fail_allocation(n) makes the
 * n-th device or pinned allocation from now on (routine workspace,
 * ddla_c_malloc, the handle's pinned word) fail as out of memory, once;
 * n <= 0 disarms.  ddla_c_live_workspaces is the number of routine workspaces
 * not yet released (0 between calls).  ddla_c_set_wait_budget sets the clock
 * budget (SM cycles; <= 0 restores the default of about 2 s) after which a
 * kernel's wait on another CTA's flag gives up and the routine reports a
 * timeout, on the handle's device. */
int ddla_c_fail_allocation(long long nth);
long long ddla_c_live_workspaces(void);
int ddla_c_set_wait_budget(void* handle, long long cycles);
void ddla_c_profile_enable(int on);
int ddla_c_profile_read(int kind, double* ms, long long* launches, double* flops, double* bytes, int reset);

#ifdef __cplusplus
}
#endif

#endif
