// ddla::ppotrf / ppotrs / pposv / pdiag_logdet on a P x Q process grid, one rank
// per GPU (src/Cholesky/ppotrf.cpp:55-323, src/PBLAS/ptrtrs.cpp:156-237,
// src/PBLAS/pdiag_logdet.cpp:11-48).
//
// Right-looking block Cholesky over the descriptor's nb x nb blocks.  Step k
// (global columns k0 .. k0+w-1, 'L'):
//   1. the owner of the diagonal block factors it in place (the 1x1 path's
//      kernels); its info word goes to every rank, and a failed pivot ends the
//      factorization on every rank with info = k0 + (the block's info);
//   2. the ranks of the block's process column receive the factored block and
//      solve their rows of the panel, X L_kk^H = A_ik (the fused solve);
//   3. every rank obtains the whole solved panel F in global row order: the
//      panel's process column all-gathers its pieces (one broadcast per
//      process row), then broadcasts F along each process row;
//   4. every rank applies A(i, j) -= F(i) F(j)^H to its local trailing block,
//      on the elements of the stored triangle, in one launch through the
//      block-cyclic index maps (ddlak_grid_gemm).
// 'U' (A = U^H U) runs the same steps on the L view L = U^H: the panel is U's
// block row, held by the block's process row, gathered along that row and
// conjugate-transposed into F, which is then broadcast along process columns.
// The reference moves only the panel rows each rank needs (a relay on square
// grids, pgeadd otherwise); every rank receiving the whole panel costs
// n * nb elements per step per rank and serves every grid shape and source
// offset with the same two broadcasts.
//
// The triangular solve (side 'L'; B distributed like A's rows) works by block
// rows with the same full panels (F now includes the diagonal block):
//   forward  k = 0, 1, ..:  the block row's process row solves L_kk Y_k = B_k
//            (fused solve), broadcasts Y_k down its process columns, and every
//            rank updates its rows below, B_i -= F_i Y_k;
//   backward k = .., 1, 0:  every rank forms its share of sum_{i>k} L_ik^H X_i,
//            the shares are summed onto the block row's process row
//            (reduce_sum), which applies X_k = L_kk^-H (Y_k - sum) with the
//            diagonal block's inverse (a forward solve on the identity).
// Side 'R' on a grid with more than one rank is not served (invalid_argument).
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>

#include <ddla/ddla.h>
#include <ddla/ddla_desc.h>
#include <ddla_kernels.h>

#include "ddla_stream.h"
#include "grid_comm.h"

namespace ddla {
namespace grid {

namespace {

template <class T> constexpr char tcode();
template <> constexpr char tcode<float>() { return 's'; }
template <> constexpr char tcode<double>() { return 'd'; }
template <> constexpr char tcode<std::complex<float>>() { return 'c'; }
template <> constexpr char tcode<std::complex<double>>() { return 'z'; }
template <class T> constexpr char real_code() { return (tcode<T>() == 's' || tcode<T>() == 'c') ? 's' : 'd'; }
template <class T> constexpr int reals_per() { return (tcode<T>() == 'c' || tcode<T>() == 'z') ? 2 : 1; }

using detail::Scope;

void ck(int e, const char* what) { detail::kernel_check(e, what); }

int read_int(const DdlaHandle_t& h, const int* d)
{
    detail::cuda_check(cudaMemcpyAsync(h->host_word, d, sizeof(int), cudaMemcpyDeviceToHost, h->stream),
                       "grid read-back");
    detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
    return *h->host_word;
}

int rank_of(const DdlaHandle_t& h, int row, int col)
{
    return h->major == 'C' ? col * h->nprows_ + row : row * h->npcols_ + col;
}

struct Geo {
    int P, Q, r, c, nb, rsrc, csrc;
    long long lld;
    // local count of global indices < g on process row / column coordinate q
    int rows_before(int g, int q) const { return num_loc(g, nb, q, rsrc, P); }
    int cols_before(int g, int q) const { return num_loc(g, nb, q, csrc, Q); }
    // the largest local extent over every process row and column: a staged piece of any rank fits
    std::size_t max_piece(int n) const
    {
        int m = 1;
        for (int q = 0; q < P; ++q) m = std::max(m, num_loc(n, nb, q, rsrc, P));
        for (int q = 0; q < Q; ++q) m = std::max(m, num_loc(n, nb, q, csrc, Q));
        return (std::size_t)m;
    }
    ddlak_gmap rmap(int first, int q, long long base) const { return {first, q, rsrc, P, nb, base}; }
    ddlak_gmap cmap(int first, int q, long long base) const { return {first, q, csrc, Q, nb, base}; }
};

Geo geo_of(const DdlaHandle_t& h, const int* desc)
{
    return {h->nprows_, h->npcols_, h->myprow_, h->mypcol_, desc[DDLA_MB_], desc[DDLA_RSRC_], desc[DDLA_CSRC_],
            (long long)desc[DDLA_LLD_]};
}

// The solved panel of block column k0 (width w), rows from global `from` to n,
// into F (n - from rows, leading dimension n - from, the L view: F(g - from, c) =
// L(g, k0 + c)) on every rank.  'L': the pieces are the rows >= from of local
// column block lc on process column pc; 'U': the columns >= from of local row
// block lr on process row pr, conjugate-transposed.  S stages one piece.
template <class T>
void full_panel(const DdlaHandle_t& h, const Geo& G, char uplo, int n, int k0, int w, int from, const T* A, T* S,
                T* F)
{
    detail::GridComm& comm = *h->grid;
    const char tc = tcode<T>();
    cudaStream_t st = h->stream;
    const bool lower = uplo == 'L';
    const int pr = indxg2p(k0, G.nb, G.rsrc, G.P), pc = indxg2p(k0, G.nb, G.csrc, G.Q);
    const int N = n - from;
    if (N <= 0) return;
    if (lower ? G.c == pc : G.r == pr) {
        const int members = lower ? G.P : G.Q, me = lower ? G.r : G.c;
        for (int q = 0; q < members; ++q) {
            const int first = lower ? G.rows_before(from, q) : G.cols_before(from, q);
            const int len = (lower ? G.rows_before(n, q) : G.cols_before(n, q)) - first;
            if (len <= 0) continue;  // the same on every member
            if (q == me) {
                if (lower) {
                    const T* piece = A + first + (long long)G.cols_before(k0, G.c) * G.lld;
                    ck(ddlak_grid_pack(tc, 0, len, w, piece, G.lld, S, len, st), "grid panel pack");
                } else {
                    const T* piece = A + G.rows_before(k0, G.r) + (long long)first * G.lld;
                    ck(ddlak_grid_pack(tc, 1, len, w, piece, G.lld, S, len, st), "grid panel pack");
                }
            }
            comm.bcast(lower ? Scope::Col : Scope::Row, q, S, sizeof(T) * (std::size_t)len * w, st);
            const ddlak_gmap m = lower ? G.rmap(first, q, from) : G.cmap(first, q, from);
            ck(ddlak_grid_unscatter(tc, len, w, S, len, F, N, &m, st), "grid panel unscatter");
        }
    }
    comm.bcast(lower ? Scope::Row : Scope::Col, lower ? pc : pr, F, sizeof(T) * (std::size_t)N * w, st);
}

}  // namespace

template <class T>
void ppotrf_grid(const DdlaHandle_t& h, char uplo, int n, T* A, const int* desc, int& info)
{
    info = 0;
    if (n == 0) return;
    detail::GridComm& comm = *h->grid;
    const Geo G = geo_of(h, desc);
    const char tc = tcode<T>();
    cudaStream_t st = h->stream;
    const bool lower = uplo == 'L';
    const int nb = G.nb;
    const int mloc = G.rows_before(n, G.r), nloc = G.cols_before(n, G.c);
    const std::size_t maxloc = (std::size_t)std::max(1, std::max(mloc, nloc));
    const std::size_t maxpiece = G.max_piece(n);
    const std::size_t sbytes = ddlak_potrs_workspace(nb, (int)maxloc);
    detail::DeviceScratch ws(h, detail::padded_bytes<int>(1) + detail::padded_bytes<T>((std::size_t)nb * nb) +
                                    detail::padded_bytes<T>(maxpiece * nb) +
                                    detail::padded_bytes<T>((std::size_t)n * nb) + sbytes);
    char* w8 = ws.data();
    int* dinfo = detail::take<int>(w8, 1);
    T* D = detail::take<T>(w8, (std::size_t)nb * nb);
    T* S = detail::take<T>(w8, maxpiece * nb);
    T* F = detail::take<T>(w8, (std::size_t)n * nb);
    void* swork = w8;
    const double minus_one[2] = {-1.0, 0.0}, one[2] = {1.0, 0.0};

    for (int k0 = 0; k0 < n; k0 += nb) {
        const int w = std::min(nb, n - k0);
        const int pr = indxg2p(k0, nb, G.rsrc, G.P), pc = indxg2p(k0, nb, G.csrc, G.Q);
        const int lr = G.rows_before(k0, G.r), lc = G.cols_before(k0, G.c);
        const bool owner = G.r == pr && G.c == pc;
        // 1. the diagonal block, and its info on every rank
        if (owner) ck(ddlak_potrf(tc, uplo, w, A + lr + (long long)lc * G.lld, G.lld, dinfo, st), "grid diagonal potrf");
        comm.bcast(Scope::All, rank_of(h, pr, pc), dinfo, sizeof(int), st);
        const int bi = read_int(h, dinfo);
        if (bi != 0) {
            info = k0 + bi;
            return;
        }
        const int from = k0 + w;
        if (from >= n) break;
        // 2. the panel ranks solve their pieces against the factored block
        if (lower ? G.c == pc : G.r == pr) {
            if (owner)
                detail::cuda_check(cudaMemcpy2DAsync(D, sizeof(T) * w, A + lr + (long long)lc * G.lld,
                                                     sizeof(T) * G.lld, sizeof(T) * w, w, cudaMemcpyDeviceToDevice,
                                                     st),
                                   "grid diagonal block copy");
            comm.bcast(lower ? Scope::Col : Scope::Row, lower ? pr : pc, D, sizeof(T) * (std::size_t)w * w, st);
            const int first = lower ? G.rows_before(from, G.r) : G.cols_before(from, G.c);
            const int len = (lower ? mloc : nloc) - first;
            if (len > 0) {
                T* panel = lower ? A + first + (long long)lc * G.lld : A + lr + (long long)first * G.lld;
                ck(ddlak_forward_solve(tc, uplo, lower ? 'R' : 'L', w, len, D, w, panel, G.lld, swork, sbytes, st),
                   "grid panel solve");
                if (read_int(h, static_cast<const int*>(swork)) != 0)
                    throw std::runtime_error("ppotrf: a device wait in the panel solve timed out");
            }
        }
        // 3. the whole solved panel on every rank
        full_panel<T>(h, G, uplo, n, k0, w, from, A, S, F);
        // 4. the local trailing block
        const int r0 = G.rows_before(from, G.r), c0 = G.cols_before(from, G.c);
        const int mrows = mloc - r0, ncols = nloc - c0;
        if (mrows > 0 && ncols > 0) {
            const ddlak_gmap ma = G.rmap(r0, G.r, from), mb = G.cmap(c0, G.c, from);
            const ddlak_gmap mi = G.rmap(r0, G.r, 0), mj = G.cmap(c0, G.c, 0);
            ck(ddlak_grid_gemm(tc, 'N', 'C', lower ? 1 : 2, mrows, ncols, w, minus_one, F, n - from, &ma, F, n - from,
                               &mb, one, A + r0 + (long long)c0 * G.lld, G.lld, &mi, &mj, st),
               "grid trailing update");
        }
    }
    detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
}

template <class T>
void ppotrs_grid(const DdlaHandle_t& h, char side, char uplo, int n, int nrhs, const T* A, const int* da, T* B,
                 const int* db)
{
    if (side != 'L')
        throw std::invalid_argument("ppotrs: side 'R' is served on a 1x1 grid only");
    if (n == 0 || nrhs == 0) return;
    detail::GridComm& comm = *h->grid;
    const Geo G = geo_of(h, da);
    const char tc = tcode<T>();
    cudaStream_t st = h->stream;
    const int nb = G.nb;
    const long long ldb = db[DDLA_LLD_];
    const int mloc = G.rows_before(n, G.r), nloc = G.cols_before(n, G.c);
    const int bloc = num_loc(nrhs, db[DDLA_NB_], G.c, db[DDLA_CSRC_], G.Q);  // my right-hand sides
    (void)nloc;
    const std::size_t maxpiece = G.max_piece(n);
    const std::size_t rc = (std::size_t)std::max(1, bloc);
    const std::size_t sbytes = ddlak_potrs_workspace(nb, (int)std::max<std::size_t>(rc, nb));
    detail::DeviceScratch ws(h, detail::padded_bytes<T>(maxpiece * nb) + detail::padded_bytes<T>((std::size_t)n * nb) +
                                    detail::padded_bytes<T>((std::size_t)nb * nb) +
                                    2 * detail::padded_bytes<T>((std::size_t)nb * rc) + sbytes);
    char* w8 = ws.data();
    T* S = detail::take<T>(w8, maxpiece * nb);
    T* F = detail::take<T>(w8, (std::size_t)n * nb);
    T* Winv = detail::take<T>(w8, (std::size_t)nb * nb);
    T* Y = detail::take<T>(w8, (std::size_t)nb * rc);
    T* Ssum = detail::take<T>(w8, (std::size_t)nb * rc);
    void* swork = w8;
    const double minus_one[2] = {-1.0, 0.0}, one[2] = {1.0, 0.0};
    auto solve_status = [&] {
        if (read_int(h, static_cast<const int*>(swork)) != 0)
            throw std::runtime_error("ppotrs: a device wait in the fused solve timed out");
    };
    const int blocks = (n + nb - 1) / nb;

    // forward: L Y = B
    for (int b = 0; b < blocks; ++b) {
        const int k0 = b * nb, w = std::min(nb, n - k0);
        const int pr = indxg2p(k0, nb, G.rsrc, G.P);
        full_panel<T>(h, G, uplo, n, k0, w, k0, A, S, F);
        const int N = n - k0;
        const int lr = G.rows_before(k0, G.r);
        if (G.r == pr && bloc > 0) {
            ck(ddlak_forward_solve(tc, 'L', 'L', w, bloc, F, N, B + lr, ldb, swork, sbytes, st), "grid block solve");
            solve_status();
            ck(ddlak_grid_pack(tc, 0, w, bloc, B + lr, ldb, Y, w, st), "grid block pack");
        }
        if (bloc > 0) comm.bcast(Scope::Col, pr, Y, sizeof(T) * (std::size_t)w * bloc, st);
        const int r0 = G.rows_before(k0 + w, G.r), mrows = mloc - r0;
        if (mrows > 0 && bloc > 0) {
            const ddlak_gmap ma = G.rmap(r0, G.r, k0);
            ck(ddlak_grid_gemm(tc, 'N', 'N', 0, mrows, bloc, w, minus_one, F, N, &ma, Y, w, nullptr, one, B + r0, ldb,
                               nullptr, nullptr, st),
               "grid forward update");
        }
    }
    // backward: L^H X = Y
    for (int b = blocks - 1; b >= 0; --b) {
        const int k0 = b * nb, w = std::min(nb, n - k0);
        const int pr = indxg2p(k0, nb, G.rsrc, G.P);
        full_panel<T>(h, G, uplo, n, k0, w, k0, A, S, F);
        const int N = n - k0;
        const int lr = G.rows_before(k0, G.r);
        const int r0 = G.rows_before(k0 + w, G.r), mrows = mloc - r0;
        if (bloc > 0) {
            // Ssum = -sum over my rows below the block of L_ik^H X_i (zero when I hold none)
            const ddlak_gmap ma = G.rmap(r0, G.r, k0);
            ck(ddlak_grid_gemm(tc, 'C', 'N', 0, w, bloc, std::max(0, mrows), minus_one, F, N, &ma, B + r0, ldb,
                               nullptr, nullptr, Ssum, w, nullptr, nullptr, st),
               "grid backward partial");
            comm.reduce_sum(Scope::Col, pr, Ssum, (std::size_t)w * bloc * reals_per<T>(), real_code<T>(), st);
        }
        if (G.r == pr && bloc > 0) {
            ck(ddlak_grid_pack(tc, 0, w, bloc, B + lr, ldb, Y, w, st), "grid block pack");
            ck(ddlak_grid_accumulate(real_code<T>(), (unsigned long long)w * bloc * reals_per<T>(), Ssum, Y, st),
               "grid backward sum");
            ck(ddlak_grid_identity(tc, w, Winv, w, st), "grid identity");
            ck(ddlak_forward_solve(tc, 'L', 'L', w, w, F, N, Winv, w, swork, sbytes, st), "grid block inverse");
            solve_status();
            ck(ddlak_grid_gemm(tc, 'C', 'N', 0, w, bloc, w, one, Winv, w, nullptr, Y, w, nullptr, nullptr, B + lr, ldb,
                               nullptr, nullptr, st),
               "grid backward block");
        }
    }
    detail::cuda_check(cudaStreamSynchronize(st), "stream synchronisation");
}

template <class T>
void pdiag_logdet_grid(const DdlaHandle_t& h, int n, const T* a, const int* desc, double total[5])
{
    double state[5];
    pdiag_logdet_local<T>(h, n, a, desc, h->nprows_, h->npcols_, h->myprow_, h->mypcol_, state);
    detail::DeviceScratch ws(h, detail::padded_bytes<double>(5));
    double* d = reinterpret_cast<double*>(ws.data());
    detail::cuda_check(cudaMemcpyAsync(d, state, sizeof state, cudaMemcpyHostToDevice, h->stream), "logdet state");
    h->grid->reduce_sum(Scope::All, 0, d, 5, 'd', h->stream);
    h->grid->bcast(Scope::All, 0, d, sizeof state, h->stream);
    detail::cuda_check(cudaMemcpyAsync(total, d, sizeof state, cudaMemcpyDeviceToHost, h->stream), "logdet state");
    detail::cuda_check(cudaStreamSynchronize(h->stream), "stream synchronisation");
}

#define DDLA_GRID_INST(T)                                                                                  \
    template void ppotrf_grid<T>(const DdlaHandle_t&, char, int, T*, const int*, int&);                  \
    template void ppotrs_grid<T>(const DdlaHandle_t&, char, char, int, int, const T*, const int*, T*,     \
                                 const int*);                                                            \
    template void pdiag_logdet_grid<T>(const DdlaHandle_t&, int, const T*, const int*, double*);
DDLA_GRID_INST(float)
DDLA_GRID_INST(double)
DDLA_GRID_INST(std::complex<float>)
DDLA_GRID_INST(std::complex<double>)
#undef DDLA_GRID_INST

}  // namespace grid
}  // namespace ddla
