// Limits of the T-matrix kernels (host and device code include them).
#pragma once

namespace pb {

constexpr int TM_THREADS = 256;
constexpr int TM_NMAX = 48;                     // orders (the reference allows 100)
constexpr int TM_NGAUSS = 128;                  // Gauss points per half (the reference allows 500)
constexpr int TM_NG = 2 * TM_NGAUSS;            // one node per thread
constexpr int TM_N2 = 2 * TM_NMAX;              // unknowns of one solve
constexpr int TM_NA = 64;                       // scattered polar angles (2 nummu, nummu <= 32)
constexpr int TM_NAZ = 30;                      // scattering azimuths (tmatrix.f90:142)
constexpr int TM_LBES = 1200;                   // NMAX + NNMAX2 limit of the reference (VARY)

}  // namespace pb
