// geometry.cuh -- the material index map built on the device from analytic shapes.
//
// The reference evaluates a Julia closure geometry(x, y, z) at every grid point on the host,
// one material after another, later materials overwriting earlier ones (src/util.jl:1-31,
// src/models.jl:85-98).  For shapes given as parameters (mfd_shape, include/maxwellfdtd.h)
// each thread takes one cell, tests the shapes in order and writes the index of the last one
// that covers it; a second pass finds each material's bounding box (atomic min/max), which
// the engine reads back to size the materials' compact state.  Every test is the header's
// double-precision expression, evaluated left to right without fused multiply-adds (the
// library is built with contraction off), so it matches a host evaluation of the same
// expression bit for bit.
#pragma once

#include "mfd_device.cuh"

namespace mfd {

__host__ __device__ __forceinline__ bool shape_covers(const mfd_shape& s, double x, double y, double z) {
    const double* p = s.p;
    switch (s.kind) {
        case MFD_SHAPE_BALL: {
            const double a = x - p[0], b = y - p[1], c = z - p[2];
            return (a * a + b * b) + c * c <= p[3] * p[3];
        }
        case MFD_SHAPE_BOX:
            return p[0] <= x && x <= p[1] && p[2] <= y && y <= p[3] && p[4] <= z && z <= p[5];
        case MFD_SHAPE_ELLIPSOID: {
            const double a = (x - p[0]) / p[3], b = (y - p[1]) / p[4], c = (z - p[2]) / p[5];
            return (a * a + b * b) + c * c <= 1.0;
        }
        case MFD_SHAPE_CYLINDER: {
            const double a = x - p[0], b = y - p[1];
            return a * a + b * b <= p[2] * p[2] && p[3] <= z && z <= p[4];
        }
        case MFD_SHAPE_HALFSPACE:
            return (p[0] * x + p[1] * y) + p[2] * z >= p[3];
        case MFD_SHAPE_ALL:
            return true;
        default:
            return false;
    }
}

// One thread per cell of the padded map (x fastest); 1-D and 2-D grids take the missing
// coordinates as 0 (2-D: y; 1-D: x and y).
__global__ void __launch_bounds__(256) geometry_kernel(uint8_t* __restrict__ geom, const Layout L, const mfd_shape* __restrict__ shapes,
                                                       const int nshape, const double* __restrict__ xs,
                                                       const double* __restrict__ ys, const double* __restrict__ zs) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y, iz = blockIdx.z;
    if (ix >= L.nx) return;
    const double x = xs ? xs[ix] : 0.0, y = ys ? ys[iy] : 0.0, z = zs[iz];
    int g = 0;
    for (int s = 0; s < nshape; ++s)
        if (shape_covers(shapes[s], x, y, z)) g = shapes[s].material;
    geom[ix + L.px * iy + (long long)L.sz * iz] = (uint8_t)g;
}

// Bounding box of each material's cells: box[6 (g - 1) + {0..5}] = x0, x1, y0, y1, z0, z1
// (initialised to INT_MAX / -1).
__global__ void __launch_bounds__(256) geometry_box_kernel(const uint8_t* __restrict__ geom, const Layout L, int* box) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y, iz = blockIdx.z;
    if (ix >= L.nx) return;
    const int g = geom[ix + L.px * iy + (long long)L.sz * iz];
    if (!g) return;
    int* b = box + 6 * (g - 1);
    atomicMin(b + 0, ix); atomicMax(b + 1, ix);
    atomicMin(b + 2, iy); atomicMax(b + 3, iy);
    atomicMin(b + 4, iz); atomicMax(b + 5, iz);
}

}  // namespace mfd
