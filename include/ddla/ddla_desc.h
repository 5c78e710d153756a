// ScaLAPACK int[9] descriptors and block-cyclic index maps.
//
// Field offsets, DESCINIT store semantics and the index maps have to match the
// reference exactly (include/ddla/ddla_desc.h:10-38 index maps, 51-64 field
// offsets, 102-137 ddlaDescInit) so that a caller's descriptor arrays drop in
// unchanged.  On the 1x1 grid every map is the identity and LLD_ is the
// leading dimension of the whole matrix.
#ifndef DDLA_DESC_H
#define DDLA_DESC_H

#include <algorithm>

#include <ddla/ddla_handle_t.h>

namespace ddla {

inline int indxg2p(int indxglob, int nb, int isrcproc, int nprocs) { return (isrcproc + indxglob / nb) % nprocs; }
inline int indxg2l(int indxglob, int nb, int nprocs) { return nb * (indxglob / (nb * nprocs)) + indxglob % nb; }
inline int indxl2g(int indxloc, int nb, int iproc, int isrcproc, int nprocs)
{
    return nprocs * nb * (indxloc / nb) + indxloc % nb + ((nprocs + iproc - isrcproc) % nprocs) * nb;
}

// Entries of an n-long index range that process iproc owns (block size nb).
inline int num_loc(int n, int nb, int iproc, int srcproc, int nprocs)
{
    const int dist = (iproc + nprocs - srcproc) % nprocs;
    int count = n / (nb * nprocs) * nb;
    const int rest = n % (nb * nprocs);
    if (rest > nb * dist) count += std::min(nb, rest - nb * dist);
    return count;
}

constexpr int DDLA_DTYPE_ = 0;
constexpr int DDLA_CTXT_ = 1;
constexpr int DDLA_M_ = 2;
constexpr int DDLA_N_ = 3;
constexpr int DDLA_MB_ = 4;
constexpr int DDLA_NB_ = 5;
constexpr int DDLA_RSRC_ = 6;
constexpr int DDLA_CSRC_ = 7;
constexpr int DDLA_LLD_ = 8;
constexpr int DDLA_DLEN_ = 9;
constexpr int DDLA_BLOCK_CYCLIC_2D = 1;

// DESCINIT: LLD_ is stored as max(lld, max(1, LOCr(M))); a negative lld derives it.
inline ddlaStatus_t ddlaDescInit(int* desc, const DdlaHandle_t& handle, int m, int n, int mb, int nb, int irsrc,
                                 int icsrc, int lld = -1)
{
    if (desc == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (handle == nullptr) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    int nprows = 0, npcols = 0, myprow = -1, mypcol = -1;
    ddlaGetGridDims(handle, nprows, npcols);
    ddlaGetGridCoords(handle, myprow, mypcol);
    if (nprows <= 0 || npcols <= 0) return ddlaStatus_t::DDLA_STATUS_INVALID_HANDLE;
    if (m < 0 || n < 0 || mb <= 0 || nb <= 0) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    if (irsrc < 0 || irsrc >= nprows || icsrc < 0 || icsrc >= npcols) return ddlaStatus_t::DDLA_STATUS_INVALID_VALUE;
    const int lld_min = std::max(1, num_loc(m, mb, myprow, irsrc, nprows));
    desc[DDLA_DTYPE_] = DDLA_BLOCK_CYCLIC_2D;
    desc[DDLA_CTXT_] = 0;
    desc[DDLA_M_] = m;
    desc[DDLA_N_] = n;
    desc[DDLA_MB_] = mb;
    desc[DDLA_NB_] = nb;
    desc[DDLA_RSRC_] = irsrc;
    desc[DDLA_CSRC_] = icsrc;
    desc[DDLA_LLD_] = std::max(lld, lld_min);
    return ddlaStatus_t::DDLA_STATUS_SUCCESS;
}

inline int indx_g2l_r(const int* desc, const DdlaHandle_t& handle, int gindx)
{
    if (handle == nullptr) return -1;
    int pr, pc, r, c;
    ddlaGetGridDims(handle, pr, pc);
    ddlaGetGridCoords(handle, r, c);
    if (r != indxg2p(gindx, desc[DDLA_MB_], desc[DDLA_RSRC_], pr) || gindx >= desc[DDLA_M_]) return -1;
    return indxg2l(gindx, desc[DDLA_MB_], pr);
}
inline int indx_g2l_c(const int* desc, const DdlaHandle_t& handle, int gindx)
{
    if (handle == nullptr) return -1;
    int pr, pc, r, c;
    ddlaGetGridDims(handle, pr, pc);
    ddlaGetGridCoords(handle, r, c);
    if (c != indxg2p(gindx, desc[DDLA_NB_], desc[DDLA_CSRC_], pc) || gindx >= desc[DDLA_N_]) return -1;
    return indxg2l(gindx, desc[DDLA_NB_], pc);
}
inline int indx_l2g_r(const int* desc, const DdlaHandle_t& handle, int lindx)
{
    if (handle == nullptr) return -1;
    int pr, pc, r, c;
    ddlaGetGridDims(handle, pr, pc);
    ddlaGetGridCoords(handle, r, c);
    return indxl2g(lindx, desc[DDLA_MB_], r, desc[DDLA_RSRC_], pr);
}
inline int indx_l2g_c(const int* desc, const DdlaHandle_t& handle, int lindx)
{
    if (handle == nullptr) return -1;
    int pr, pc, r, c;
    ddlaGetGridDims(handle, pr, pc);
    ddlaGetGridCoords(handle, r, c);
    return indxl2g(lindx, desc[DDLA_NB_], c, desc[DDLA_CSRC_], pc);
}

}  // namespace ddla

#endif
