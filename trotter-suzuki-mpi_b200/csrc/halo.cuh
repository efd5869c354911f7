// Periodic halo refresh of one tile (src/cpukernel.cpp:706-716,738-746, one
// process): x-halo columns of rows [xr0, xr1) take the opposite inner
// columns (the reference: [iy0, iy0 + H - 2*hy)), then y-halo rows take the
// opposite inner rows (all columns).
// Each destination cell is written from the cell its value ends up coming
// from; those source cells are never destinations, so one pass suffices.
#pragma once
#include "step_kernel.cuh"

namespace tsb {

// Destination cells of the halo refresh.
__host__ __device__ inline int halo_cell_count(int W, int H, int hx, int hy, int px, int py) {
    const int nx = px ? 2 * hx * H : 0;
    const int ny = py ? 2 * hy * (px ? W - 2 * hx : W) : 0;
    return nx + ny;
}

// Destination cells k0, k0 + stride, ... of the refresh.
template <typename T>
__device__ __forceinline__ void halo_cells(Cx<T> *psi, int W, int H, int P, int hx, int hy, int px,
                                           int py, int xr0, int xr1, int k0, int stride) {
    const int nx_dest = px ? 2 * hx * H : 0;
    const int ncols_b = px ? W - 2 * hx : W;  // y-halo cells outside the x-halo columns
    const int n = halo_cell_count(W, H, hx, hy, px, py);
    const int Nx = W - 2 * hx, Ny = H - 2 * hy;
    for (int k = k0; k < n; k += stride) {
        int x, y;
        if (k < nx_dest) {
            y = k / (2 * hx);
            const int c = k % (2 * hx);
            x = c < hx ? c : W - 2 * hx + c;
        } else {
            const int kk = k - nx_dest;
            const int rr = kk / ncols_b, c = kk % ncols_b;
            y = rr < hy ? rr : H - 2 * hy + rr;
            x = px ? hx + c : c;
        }
        int ys = y;
        if (py) {
            if (y < hy) ys = y + Ny;
            else if (y >= H - hy) ys = y - Ny;
        }
        int xs = x;
        if (px && ys >= xr0 && ys < xr1) {
            if (x < hx) xs = x + Nx;
            else if (x >= W - hx) xs = x - Nx;
        }
        if (xs == x && ys == y) continue;
        psi[(size_t)y * P + x] = psi[(size_t)ys * P + xs];
    }
}

}  // namespace tsb
