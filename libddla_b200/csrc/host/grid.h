// Distributed routines on a grid of more than one rank (grid.cpp).
#pragma once
#include <ddla/ddla.h>

namespace ddla {
namespace grid {

template <class T>
void ppotrf_grid(const DdlaHandle_t& h, char uplo, int n, T* A, const int* desc, int& info);
template <class T>
void ppotrs_grid(const DdlaHandle_t& h, char side, char uplo, int n, int nrhs, const T* A, const int* da, T* B,
                 const int* db);
// the five summed pdiag_logdet states of every rank, on every rank
template <class T>
void pdiag_logdet_grid(const DdlaHandle_t& h, int n, const T* a, const int* desc, double total[5]);

}  // namespace grid
}  // namespace ddla
