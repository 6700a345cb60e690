// Interleaved-storage kernels (quad.cuh) for the Lat_square_1 lattice table, in a translation unit of their own.
#define SCK_QUAD_KERNELS
#include "quad.cuh"

SCK_QUAD_INSTANTIATE(sck::Lat_square_1)
