// C ABI of the B200 Trotter-Suzuki kernel (include/ts_b200.h).
//
// Host side: one handle per tile.  It owns two device tiles (the step reads
// one and writes the other, as the reference's double buffer
// p_real[.][sense], src/cpukernel.cpp:244-247), the exponential table, the
// rotation coefficient tables, reduction scratch and a CUDA stream.  Work is
// only queued; nothing synchronises the host except the calls that return
// data.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>

#include "step_kernel.cuh"
#include "handle.h"
#include "halo.cuh"
#include "step_launch.h"
#include "step2_decl.h"
#include "ts_b200.h"

using tsb::Cx;
using tsb::Scalars;
using tsb::StepArgs;

namespace tsbh {
std::atomic<uint64_t> g_launches{0};
}  // namespace tsbh
using tsbh::g_launches;

namespace {


// ------------------------------------------------ FP32 rounding of rotations
// The FP32 step works in delta form (see step_kernel.cuh): a 2x2 rotation
// with coefficients (a, b) is stored as (a - 1, b).  It conserves the norm
// only if (1 + am1)^2 + b^2 = 1 for the stored floats.  Among the floats within
// `span` ulps of the rounded values the pair with the smallest defect
// |2 am1 + am1^2 + b^2| (exact in double for float inputs) is kept; ties go to
// the pair closest to the exact values.  am1 is passed in double, computed
// without cancellation by the caller.
__host__ __device__ inline void unimodular_float_pair(double am1, double b, int span, float *fa,
                                                      float *fb) {
    const float a0 = (float)am1, b0 = (float)b;
    float ba = a0, bb = b0;
    auto defect = [](float x, float y) {
        return fabs(2.0 * (double)x + (double)x * x + (double)y * y);
    };
    double best = defect(a0, b0);
    double bestd = fabs((double)a0 - am1) + fabs((double)b0 - b);
    float ai = a0;
    for (int i = 0; i < span; ++i) ai = nextafterf(ai, -INFINITY);
    for (int i = -span; i <= span; ++i, ai = nextafterf(ai, INFINITY)) {
        float bj = b0;
        for (int j = 0; j < span; ++j) bj = nextafterf(bj, -INFINITY);
        for (int j = -span; j <= span; ++j, bj = nextafterf(bj, INFINITY)) {
            const double err = defect(ai, bj);
            const double d = fabs((double)ai - am1) + fabs((double)bj - b);
            if (err < best || (err == best && d < bestd)) {
                best = err;
                bestd = d;
                ba = ai;
                bb = bj;
            }
        }
    }
    *fa = ba;
    *fb = bb;
}

// The same objective as unimodular_float_pair (smallest defect, then the
// closest pair) in a fraction of the work, for tables rebuilt every step.  For
// each float b_j within `span` ulps of round(b), the exact unimodular partner
// a(b_j) is followed from (am1, b) along the circle to second order
// (da = -b/(1+a) db - db^2 / (2 (1+a)^3), from (1+a)^2 + b^2 = 1), and only the
// two floats bracketing it are scored: 2a + a^2 is monotone there, so they
// hold the smallest defect over ALL floats a for that b_j (a superset of the
// exhaustive search's candidates).  Near |angle| = pi/2 (|1 + am1| < 1/4) the
// expansion is not used and the exhaustive search runs instead.
__host__ __device__ inline void unimodular_float_pair_fast(double am1, double b, int span,
                                                           float *fa, float *fb) {
    const double c = 1.0 + am1;
    if (!(fabs(c) >= 0.25)) {
        unimodular_float_pair(am1, b, span, fa, fb);
        return;
    }
    const double inv = 1.0 / c;
    auto defect = [](float x, float y) {
        return fabs(2.0 * (double)x + (double)x * x + (double)y * y);
    };
    const float b0 = (float)b;
    float ba = (float)am1, bb = b0;
    double best = defect(ba, bb);
    double bestd = fabs((double)ba - am1) + fabs((double)bb - b);
    float bj = b0;
    for (int j = 0; j < span; ++j) bj = nextafterf(bj, -INFINITY);
    for (int j = -span; j <= span; ++j, bj = nextafterf(bj, INFINITY)) {
        const double db = (double)bj - b;
        const double am = am1 - b * inv * db - 0.5 * inv * inv * inv * db * db;
        const float a1 = (float)am;
        const float a2 = nextafterf(a1, (double)a1 < am ? INFINITY : -INFINITY);
        for (int t = 0; t < 2; ++t) {
            const float ai = t ? a2 : a1;
            const double err = defect(ai, bj);
            const double d = fabs((double)ai - am1) + fabs((double)bj - b);
            if (err < best || (err == best && d < bestd)) {
                best = err;
                bestd = d;
                ba = ai;
                bb = bj;
            }
        }
    }
    *fa = ba;
    *fb = bb;
}

// cos(k) - 1 and cosh(k) - 1 without cancellation.
__host__ __device__ inline double cos_m1(double k) {
    const double h = sin(0.5 * k);
    return -2.0 * h * h;
}
__host__ __device__ inline double cosh_m1(double k) {
    const double h = sinh(0.5 * k);
    return 2.0 * h * h;
}

// ------------------------------------------------------------------ kernels

// Interleave host-order SoA doubles (row stride `sstride`) into the device
// AoS tile of type T (row pitch P); padding columns [W, P) are zeroed.
template <typename T>
__global__ void pack_state_kernel(Cx<T> *dst, int W, int H, int P, const double *re,
                                  const double *im, size_t sstride) {
    const size_t n = (size_t)P * H;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(k / P), x = (int)(k % P);
        Cx<T> v{T(0), T(0)};
        if (x < W) {
            v.re = (T)re[(size_t)y * sstride + x];
            v.im = (T)im[(size_t)y * sstride + x];
        }
        dst[k] = v;
    }
}

// Table: Cx<T> per cell in real time, T (real part only) in imaginary time.
template <typename T>
__global__ void pack_table_kernel(void *dst, int imag, int W, int H, int P, const double *re,
                                  const double *im, size_t sstride) {
    const size_t n = (size_t)P * H;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(k / P), x = (int)(k % P);
        const double vr = x < W ? re[(size_t)y * sstride + x] : 0.0;
        const double vi = x < W ? im[(size_t)y * sstride + x] : 0.0;
        if (imag) {
            reinterpret_cast<T *>(dst)[k] = (T)vr;
        } else if (sizeof(T) == 4) {
            // delta form (cos - 1, sin); vr - 1 is exact enough in double
            float fr, fi;
            unimodular_float_pair(vr - 1.0, vi, 4, &fr, &fi);
            reinterpret_cast<Cx<T> *>(dst)[k] = Cx<T>{(T)fr, (T)fi};
        } else {
            reinterpret_cast<Cx<T> *>(dst)[k] = Cx<T>{(T)vr, (T)vi};
        }
    }
}

using tsb::kSmallAngle;
using tsb::small_angle_sincos;

// The table from a potential on the device: exp(-i dt V) in real time
// ((cos - 1, -sin) in float: delta form, pair chosen by the fast search),
// exp(-dt V) in imaginary time; the host path tabulates the same with
// std::exp(complex) (src/solver.cpp:74-109).  V: W x H doubles, row pitch vp.
// One thread per cell of a row (blockIdx.y strides over the rows): no index
// division, coalesced in both arrays.
template <typename T>
__global__ void table_from_potential_kernel(void *dst, int imag, int W, int H, int P,
                                            const double *V, size_t vp, double dt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= P) return;
    for (int y = blockIdx.y; y < H; y += gridDim.y) {
        const size_t k = (size_t)y * P + x;
        const double ang = x < W ? dt * V[(size_t)y * vp + x] : 0.0;
        if (imag) {
            reinterpret_cast<T *>(dst)[k] = x < W ? (T)exp(-ang) : T(0);
            continue;
        }
        double s, cm1;
        if (fabs(ang) <= kSmallAngle) {
            small_angle_sincos(ang, &s, &cm1);
        } else {
            double c;
            sincos(ang, &s, &c);
            cm1 = sizeof(T) == 4 ? cos_m1(ang) : c - 1.0;
            if (sizeof(T) == 8) {
                reinterpret_cast<Cx<T> *>(dst)[k] =
                    x < W ? Cx<T>{(T)c, (T)-s} : Cx<T>{T(0), T(0)};
                continue;
            }
        }
        if (sizeof(T) == 4) {
            float fr, fi;
            // span 1: about the defect of the exhaustive span-4 search at a
            // sixth of the FP64 work of span 4, for a table made every step
            unimodular_float_pair_fast(x < W ? cm1 : -1.0, x < W ? -s : 0.0, 1, &fr, &fi);
            reinterpret_cast<Cx<T> *>(dst)[k] = Cx<T>{(T)fr, (T)fi};
        } else {
            reinterpret_cast<Cx<T> *>(dst)[k] =
                x < W ? Cx<T>{(T)(1.0 + cm1), (T)-s} : Cx<T>{T(0), T(0)};
        }
    }
}

void launch_table_from_potential(ts_b200_kernel *k, const double *V, size_t vp, double dt) {
    const dim3 grid((k->P + 255) / 256, std::min(k->H, 65535));
    if (k->fp32)
        table_from_potential_kernel<float><<<grid, 256, 0, k->stream>>>(
            k->tab, k->imag ? 1 : 0, k->W, k->H, k->P, V, vp, dt);
    else
        table_from_potential_kernel<double><<<grid, 256, 0, k->stream>>>(
            k->tab, k->imag ? 1 : 0, k->W, k->H, k->P, V, vp, dt);
}

// De-interleave a w x h window at (x0, y0) into SoA doubles with stride w,
// multiplying by `scale` (the pending imaginary-time renormalisation).
template <typename T>
__global__ void unpack_state_kernel(const Cx<T> *src, int P, int x0, int y0, int w, int h,
                                    const Scalars *scal, int use_scale, double *re, double *im) {
    const double s = use_scale ? scal->pending_inv : 1.0;
    const size_t n = (size_t)w * h;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(k / w), x = (int)(k % w);
        const Cx<T> v = src[(size_t)(y0 + y) * P + (x0 + x)];
        re[k] = (double)v.re * s;
        im[k] = (double)v.im * s;
    }
}

// Copy the tile with a pitch change, optionally folding in the pending scale.
template <typename T>
__global__ void copy_tile_kernel(Cx<T> *dst, size_t dpitch, const Cx<T> *src, size_t spitch,
                                 int W, int H, const Scalars *scal, int use_scale) {
    const T s = use_scale ? (T)scal->pending_inv : T(1);
    const size_t n = (size_t)W * H;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(k / W), x = (int)(k % W);
        Cx<T> v = src[(size_t)y * spitch + x];
        if (use_scale) {
            v.re *= s;
            v.im *= s;
        }
        dst[(size_t)y * dpitch + x] = v;
    }
}

// Periodic halo refresh (src/cpukernel.cpp:706-716,738-746, one process):
// x-halo columns of rows [iy0, iy0 + H - 2*hy) take the opposite inner
// columns, then y-halo rows take the opposite inner rows (all columns).  Each
// destination cell is written from the cell its value ends up coming from;
// those source cells are never destinations, so one pass suffices.
template <typename T>
__global__ void halo_kernel(Cx<T> *psi, int W, int H, int P, int hx, int hy, int px, int py,
                            int xr0, int xr1) {
    tsb::halo_cells(psi, W, H, P, hx, hy, px, py, xr0, xr1, blockIdx.x * blockDim.x + threadIdx.x,
                    gridDim.x * blockDim.x);
}

// -------------------------------------------------------------- reductions
// Deterministic FP64 reductions over the inner region: a fixed grid, each
// thread walks a fixed set of cells, a fixed block tree, then the last block
// to finish sums the block partials in order.
constexpr int RED_THREADS = 256;
constexpr int RED_MAX_BLOCKS = 1184;  // 8 per SM on a 148-SM B200
constexpr int RED_MAX_TERMS = 10;

struct RedArgs {
    const void *psi;
    int W, H, P;
    int ix0, ix1, iy0, iy1;
    const Scalars *scal;
    int use_scale;
    const double *V;
    double dx, dy;
    int start_x, start_y, gnx, gny;
    double Lx, Ly;
    double mass, g, glhy, omega;
    int cyl;           // cylindrical lattice: radial coordinates, energy region from column 3
    double *partials;  // gridDim.x * RED_MAX_TERMS
    double *out;       // RED_MAX_TERMS
    unsigned int *ticket;
};

// Cell-centre coordinates (src/common.cpp:45-81): cartesian, or on a
// cylindrical lattice the radial x from the tile's edge, r = -dx/2 at column 0.
__device__ __forceinline__ void cell_coords(const RedArgs &a, int xi, int yi, double *xo,
                                            double *yo) {
    if (a.cyl) {
        double idy = __dadd_rn(__dadd_rn(__dmul_rn(a.start_y, a.dy), __dmul_rn(0.5, a.dy)),
                               __dmul_rn(yi, a.dy));
        const double idx = __dsub_rn(__dadd_rn(__dmul_rn(a.start_x, a.dx), __dmul_rn(xi, a.dx)),
                                     __dmul_rn(0.5, a.dx));
        const double y_c = __dmul_rn(__dmul_rn(a.gny, a.dy), 0.5);
        if (idy - y_c < -a.Ly * 0.5) idy = __dadd_rn(idy, a.Ly);
        if (idy - y_c > a.Ly * 0.5) idy = __dsub_rn(idy, a.Ly);
        *xo = idx;
        *yo = __dsub_rn(idy, y_c);
        return;
    }
    double idy = __dadd_rn(__dadd_rn(__dmul_rn(a.start_y, a.dy), __dmul_rn(0.5, a.dy)),
                           __dmul_rn(yi, a.dy));
    double idx = __dadd_rn(__dadd_rn(__dmul_rn(a.start_x, a.dx), __dmul_rn(0.5, a.dx)),
                           __dmul_rn(xi, a.dx));
    const double x_c = __dmul_rn(__dmul_rn(a.gnx, a.dx), 0.5);
    const double y_c = __dmul_rn(__dmul_rn(a.gny, a.dy), 0.5);
    if (idx - x_c < -a.Lx * 0.5) idx = __dadd_rn(idx, a.Lx);
    if (idx - x_c > a.Lx * 0.5) idx = __dsub_rn(idx, a.Lx);
    if (idy - y_c < -a.Ly * 0.5) idy = __dadd_rn(idy, a.Ly);
    if (idy - y_c > a.Ly * 0.5) idy = __dsub_rn(idy, a.Ly);
    *xo = __dsub_rn(idx, x_c);
    *yo = __dsub_rn(idy, y_c);
}

template <typename T>
__device__ __forceinline__ Cx<double> ldc(const RedArgs &a, double s, int x, int y) {
    const Cx<T> v = reinterpret_cast<const Cx<T> *>(a.psi)[(size_t)y * a.P + x];
    return Cx<double>{(double)v.re * s, (double)v.im * s};
}

template <int NT>
__device__ void block_reduce_and_finish(const RedArgs &a, double (&acc)[NT]) {
    __shared__ double sh[RED_THREADS];
    __shared__ unsigned int s_last;
    for (int t = 0; t < NT; ++t) {
        sh[threadIdx.x] = acc[t];
        __syncthreads();
        for (int h = RED_THREADS / 2; h > 0; h >>= 1) {
            if ((int)threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) a.partials[blockIdx.x * RED_MAX_TERMS + t] = sh[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int k = atomicAdd(a.ticket, 1u);
        s_last = (k == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (s_last && threadIdx.x < NT) {
        __threadfence();
        double s = 0.0;
        for (unsigned int b = 0; b < gridDim.x; ++b)
            s += __ldcg(&a.partials[b * RED_MAX_TERMS + threadIdx.x]);
        a.out[threadIdx.x] = s;
    }
    if (s_last && threadIdx.x == 0) *a.ticket = 0u;
}

// Squared norm of the inner region (src/cpukernel.cpp:526-549).
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) norm_kernel(RedArgs a) {
    const double s = a.use_scale ? a.scal->pending_inv : 1.0;
    const int w = a.ix1 - a.ix0;
    const size_t n = (size_t)w * (a.iy1 - a.iy0);
    double acc[1] = {0.0};
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int y = a.iy0 + (int)(k / w), x = a.ix0 + (int)(k % w);
        const Cx<double> c = ldc<T>(a, s, x, y);
        acc[0] += c.re * c.re + c.im * c.im;
    }
    block_reduce_and_finish<1>(a, acc);
}

// Energy sums of src/solver.cpp:320-420 (single component, cartesian):
// [0] norm2, [1] norm2 over the kinetic region, [2] kinetic, [3] potential,
// [4] rotational, [5] intra-species, [6] Lee-Huang-Yang.
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) energy_kernel(RedArgs a) {
    const double s = a.use_scale ? a.scal->pending_inv : 1.0;
    const int w = a.ix1 - a.ix0;
    const size_t n = (size_t)w * (a.iy1 - a.iy0);
    const int ihx = a.ix0, ihy = a.iy0, ehx = a.W - a.ix1, ehy = a.H - a.iy1;
    const double cost_E = -1. / (2. * a.mass);
    const double c1 = -1. / 12., c2 = 4. / 3., c3 = -2.5;
    const double d1 = 1. / 6., d2 = -1., d3 = 0.5, d4 = 1. / 3.;
    const double idx2 = 1.0 / (a.dx * a.dx), idy2 = 1.0 / (a.dy * a.dy);
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = a.iy0 + (int)(k / w), j = a.ix0 + (int)(k % w);
        const Cx<double> c = ldc<T>(a, s, j, i);
        const double n2 = c.re * c.re + c.im * c.im;
        acc[0] += n2;
        acc[3] += n2 * a.V[(size_t)i * a.W + j];
        acc[5] += n2 * n2 * 0.5 * a.g;
        if (a.glhy != 0.0) acc[6] += pow(n2, 2.5) * 0.4 * a.glhy;
        // src/solver.cpp:301,358-361: on a cylindrical lattice the kinetic
        // region starts 3 columns further from the axis
        if (((i - a.iy0 >= (ihy == 0) * 2 && i < a.iy1 - (ehy == 0) * 2) || a.H == 1) &&
            (j - a.ix0 >= (ihx == 0) * 2 + (a.cyl ? 3 : 0) && j < a.ix1 - (ehx == 0) * 2)) {
            const Cx<double> r = ldc<T>(a, s, j + 1, i), l = ldc<T>(a, s, j - 1, i);
            const Cx<double> rr = ldc<T>(a, s, j + 2, i), ll = ldc<T>(a, s, j - 2, i);
            acc[1] += n2;
            // Re(conj(c) * lap) with lap the 4th-order 5-point Laplacian
            const double lre = c1 * rr.re + c2 * r.re + c2 * l.re + c1 * ll.re + c3 * c.re;
            const double lim = c1 * rr.im + c2 * r.im + c2 * l.im + c1 * ll.im + c3 * c.im;
            acc[2] += cost_E * (c.re * lre + c.im * lim) * idx2;
            if (a.H > 1) {
                const Cx<double> up = ldc<T>(a, s, j, i - 1), dn = ldc<T>(a, s, j, i + 1);
                const Cx<double> uu = ldc<T>(a, s, j, i - 2), dd = ldc<T>(a, s, j, i + 2);
                const double yre = c1 * dd.re + c2 * dn.re + c2 * up.re + c1 * uu.re + c3 * c.re;
                const double yim = c1 * dd.im + c2 * dn.im + c2 * up.im + c1 * uu.im + c3 * c.im;
                acc[2] += cost_E * (c.re * yre + c.im * yim) * idy2;
                if (a.omega != 0.0) {
                    double x, y;
                    cell_coords(a, j, i, &x, &y);
                    // rot_x = i*y*omega/dx, rot_y = i*x*omega/dy (src/solver.cpp:384-387)
                    const double ry = x * a.omega / a.dy, rx = y * a.omega / a.dx;
                    const double dyre = d4 * up.re + d3 * c.re + d2 * dn.re + d1 * dd.re;
                    const double dyim = d4 * up.im + d3 * c.im + d2 * dn.im + d1 * dd.im;
                    const double dxre = d4 * r.re + d3 * c.re + d2 * l.re + d1 * ll.re;
                    const double dxim = d4 * r.im + d3 * c.im + d2 * l.im + d1 * ll.im;
                    // inner = i*ry*dy_ + i*rx*dx_ ; Re(conj(c) * inner)
                    const double inre = -(ry * dyim + rx * dxim);
                    const double inim = ry * dyre + rx * dxre;
                    acc[4] += c.re * inre + c.im * inim;
                }
            }
        }
    }
    block_reduce_and_finish<7>(a, acc);
}

// Expectation-value sums of src/model.cpp:405-455 (2D cartesian):
// [0] norm2 [1] x [2] y [3] xx [4] yy [5] px [6] py [7] pxpx [8] pypy [9] lz
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) expect_kernel(RedArgs a) {
    const double s = a.use_scale ? a.scal->pending_inv : 1.0;
    const int w = a.ix1 - a.ix0;
    const size_t n = (size_t)w * (a.iy1 - a.iy0);
    const int ihx = a.ix0, ihy = a.iy0, ehx = a.W - a.ix1, ehy = a.H - a.iy1;
    const double c1 = -1. / 12., c2 = 4. / 3., c3 = -2.5;
    const double d1 = 1. / 6., d2 = -1., d3 = 0.5, d4 = 1. / 3.;
    double acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = a.iy0 + (int)(k / w), j = a.ix0 + (int)(k % w);
        const Cx<double> c = ldc<T>(a, s, j, i);
        double x, y;
        cell_coords(a, j, i, &x, &y);
        const double n2 = c.re * c.re + c.im * c.im;
        acc[0] += n2;
        acc[1] += n2 * x;
        acc[2] += n2 * y;
        acc[3] += n2 * x * x;
        acc[4] += n2 * y * y;
        if (i - ihy >= (ihy == 0) * 2 && i < a.iy1 - (ehy == 0) * 2 && j - ihx >= (ihx == 0) * 2 &&
            j < a.ix1 - (ehx == 0) * 2) {
            const Cx<double> up = ldc<T>(a, s, j, i - 1), dn = ldc<T>(a, s, j, i + 1);
            const Cx<double> r = ldc<T>(a, s, j + 1, i), l = ldc<T>(a, s, j - 1, i);
            const Cx<double> uu = ldc<T>(a, s, j, i - 2), dd = ldc<T>(a, s, j, i + 2);
            const Cx<double> rr = ldc<T>(a, s, j + 2, i), ll = ldc<T>(a, s, j - 2, i);
            const double dxre = d4 * r.re + d3 * c.re + d2 * l.re + d1 * ll.re;
            const double dxim = d4 * r.im + d3 * c.im + d2 * l.im + d1 * ll.im;
            const double dyre = d4 * up.re + d3 * c.re + d2 * dn.re + d1 * dd.re;
            const double dyim = d4 * up.im + d3 * c.im + d2 * dn.im + d1 * dd.im;
            // Im(conj(c) * z) = c.re*z.im - c.im*z.re ; Re(conj(c)*z) = c.re*z.re + c.im*z.im
            acc[5] += c.re * dxim - c.im * dxre;
            acc[6] += c.re * dyim - c.im * dyre;
            const double lxre = c1 * rr.re + c2 * r.re + c2 * l.re + c1 * ll.re + c3 * c.re;
            const double lxim = c1 * rr.im + c2 * r.im + c2 * l.im + c1 * ll.im + c3 * c.im;
            const double lyre = c1 * dd.re + c2 * dn.re + c2 * up.re + c1 * uu.re + c3 * c.re;
            const double lyim = c1 * dd.im + c2 * dn.im + c2 * up.im + c1 * uu.im + c3 * c.im;
            acc[7] += c.re * lxre + c.im * lxim;
            acc[8] += c.re * lyre + c.im * lyim;
            const double zre = y / a.dx * dxre + x / a.dy * dyre;
            const double zim = y / a.dx * dxim + x / a.dy * dyim;
            acc[9] += c.re * zim - c.im * zre;
        }
    }
    block_reduce_and_finish<10>(a, acc);
}

// --------------------------------------------------------- step dispatch
// The step variants are instantiated in step_f64_real.cu, step_f64_imag.cu,
// step_f32_real.cu and step_f32_imag.cu (compiled in parallel).
// w2 > 0: the look-ahead walk (walk2.cuh) with w2 rows per iteration, else
// the checked walk (step_kernel.cuh)
template <typename T>
cudaError_t dispatch_step(int C, bool imag, bool rot, int phase, int w2, const StepArgs<T> &a,
                          int warps, size_t smem, int blocks, cudaStream_t st, int *bps,
                          bool pdl = false);

template <>
cudaError_t dispatch_step<double>(int C, bool imag, bool rot, int phase, int w2,
                                  const StepArgs<double> &a, int warps, size_t smem, int blocks,
                                  cudaStream_t st, int *bps, bool pdl) {
    if (w2 && (phase == 3 || phase == 7))
        return imag ? tsb::launch_step2pair_f64_imag(w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2pair_f64_real(w2, phase, a, warps, smem, blocks, st, bps, pdl);
    if (w2 && phase >= 4 && phase <= 6)
        return imag ? tsb::launch_step2cyl_f64_imag(w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2cyl_f64_real(w2, phase, a, warps, smem, blocks, st, bps, pdl);
    if (w2 && rot)
        return imag ? tsb::launch_step2rot_f64_imag(C, w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2rot_f64_real(C, w2, phase, a, warps, smem, blocks, st, bps, pdl);
    if (w2)
        return imag ? tsb::launch_step2_f64_imag(C, w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2_f64_real(C, w2, phase, a, warps, smem, blocks, st, bps, pdl);
    return imag ? tsb::launch_step_f64_imag(C, rot, phase, a, warps, smem, blocks, st, bps)
                : tsb::launch_step_f64_real(C, rot, phase, a, warps, smem, blocks, st, bps);
}

template <>
cudaError_t dispatch_step<float>(int C, bool imag, bool rot, int phase, int w2,
                                 const StepArgs<float> &a, int warps, size_t smem, int blocks,
                                 cudaStream_t st, int *bps, bool pdl) {
    if (w2 && (phase == 3 || phase == 7))
        return imag ? tsb::launch_step2pair_f32_imag(w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2pair_f32_real(w2, phase, a, warps, smem, blocks, st, bps, pdl);
    if (w2 && phase >= 4 && phase <= 6)
        return imag ? tsb::launch_step2cyl_f32_imag(w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2cyl_f32_real(w2, phase, a, warps, smem, blocks, st, bps, pdl);
    if (w2 && rot)
        return imag ? tsb::launch_step2rot_f32_imag(C, w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2rot_f32_real(C, w2, phase, a, warps, smem, blocks, st, bps, pdl);
    if (w2)
        return imag ? tsb::launch_step2_f32_imag(C, w2, phase, a, warps, smem, blocks, st, bps, pdl)
                    : tsb::launch_step2_f32_real(C, w2, phase, a, warps, smem, blocks, st, bps, pdl);
    return imag ? tsb::launch_step_f32_imag(C, rot, phase, a, warps, smem, blocks, st, bps)
                : tsb::launch_step_f32_real(C, rot, phase, a, warps, smem, blocks, st, bps);
}

using tsbh::div_up;

// Shared memory of an SM and the part the runtime reserves per block (sm_100).
constexpr int kSmemPerSm = 228 * 1024;
constexpr int kSmemReservedPerBlock = 1024;
using tsbh::slot_bytes;
using tsbh::kSchedLen;

}  // namespace


namespace {

int fail(ts_b200_kernel *k, int status, const std::string &msg) {
    if (k) k->err = msg;
    return status;
}

int cuda_fail(ts_b200_kernel *k, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (k) k->err = m;
    return e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR;
}

#define TSB_CHECK(k, call)                                   \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(k, e_, #call); \
    } while (0)

void drop_graph(ts_b200_kernel *k) {
    if (k->graph) {
        cudaGraphExecDestroy(k->graph);
        k->graph = nullptr;
        k->graph_steps = 0;
    }
}

void choose_launch(ts_b200_kernel *k) {
    // Column strips of 32*C cells with C = 2: the short 2-cell rows keep the
    // register window small enough for 4 blocks of 4 warps per SM.  The
    // segment height is fixed once the resident grid is known (auto_seg).
    k->C = 2;
    k->seg_h = 64;
    k->auto_seg = true;
    k->warps = 4;
    k->ring = 4;
    // Programmatic dependent launch of each step: measured faster on 2048^2
    // in imaginary time (FP64 39.9 -> 38.6 us, FP32 29.2 -> 28.4 us) and FP32
    // real time (30.1 -> 29.0 us), slower in FP64 real time (47.3 -> 48.3 us)
    k->overlap = !(k->imag == false && k->fp32 == false);
    // single precision in a rotating frame: 4 cells per lane (strips of 128
    // columns carry 112 output columns instead of 48 of 64: 8192^2 vortex
    // step 610 -> 569 us)
    if (k->rot && k->fp32 && k->walk2 > 0 && !k->cyl && k->phase <= 2) k->C = 4;
}

// A row's table is read two rows after its psi: the ring must hold those
// three rows plus at least one in flight.
int min_ring(const ts_b200_kernel *) { return 4; }

// The look-ahead walk covers every variant: phases 0-2 cartesian (in a
// rotating frame with 2 cells per lane, or 4 in single precision), one
// species of a pair (phases 3 and 7) and cylindrical lattices (phases 4-6)
// with 2 cells per lane.
bool use_walk2(const ts_b200_kernel *k) {
    if (k->walk2 <= 0) return false;
    if (k->cyl || (k->phase & 3) == 3) return k->C == 2 && !k->rot;
    return !k->rot || k->C == 2 || k->fp32;
}

// Rows of the look-ahead walk's register window and ring (8 in a rotating
// frame: its step has 6 vertical sweeps).
int walk_window(const ts_b200_kernel *k) { return k->rot ? 8 : 6; }

// Rows per iteration of the look-ahead walk in use (0: the checked walk);
// two rows per iteration exist for 2 cells per lane, and for 4 in a
// single-precision rotating frame.
int walk_rows(const ts_b200_kernel *k) {
    if (!use_walk2(k)) return 0;
    return (k->walk2 == 2 && (k->C == 2 || (k->rot && k->fp32))) ? 2 : 1;
}

// Rows per segment as launched: the look-ahead walk needs even segments
// (compile-time row parities).
int eff_seg(const ts_b200_kernel *k) { return use_walk2(k) ? (k->seg_h + 1) & ~1 : k->seg_h; }

// One round of tasks over the resident warps: as many row segments per strip
// as there are resident warps per strip.
// Rows per segment for a grid of `blocks_per_sm` blocks on every SM, one
// task per warp: every SM then holds the same number of tasks (the launch
// time is that of the most loaded SM).
int balanced_segments(const ts_b200_kernel *k, int blocks_per_sm, int warps) {
    const int hx = (k->rot || k->cyl) ? 8 : 4;  // Variant::HX
    const int wo = 32 * k->C - 2 * hx;
    const int strips = div_up(k->W, wo);
    const long rw = (long)blocks_per_sm * k->num_sms * warps;
    const int per_strip = (int)std::max(1L, rw / std::max(1, strips));
    const int seg = std::max(8, div_up(k->H, per_strip));
    return use_walk2(k) ? (seg + 1) & ~1 : seg;
}

// Default: 4 blocks of 4 warps per SM (fewer, taller tasks than a grid
// filling every resident slot: less halo work per row, the same balance),
// with segments of at most kMaxAutoSegment rows: on large tiles one task per
// warp means segments of hundreds of rows, which ran 1.3-1.6x slower than
// 64-128-row segments taken by the persistent warps in turn (8192^2 rotating
// frame: 2.02 -> 1.35 ms per step in double, 1.72 -> 1.07 in float).
constexpr int kMaxAutoSegment = 128;
void auto_segments(ts_b200_kernel *k) {
    const int bps = std::max(1, k->resident_blocks / std::max(1, k->num_sms));
    k->seg_h = std::min(kMaxAutoSegment, balanced_segments(k, std::min(4, bps), k->warps));
}

// pad: the shared memory of a launch with programmatic dependent launch
// (padded to the grid's share of blocks per SM); without it, the kernel's own
// need (for the occupancy that chooses the shape).
// part: the launch covers the part's row windows (no padding).
void geometry(const ts_b200_kernel *k, int *strips, int *segs, int *blocks, size_t *smem,
              bool pad = true, const tsbh::StepPart *part = nullptr) {
    const int hx = (k->rot || k->cyl) ? 8 : 4;  // Variant::HX
    const int wo = 32 * k->C - 2 * hx;
    *strips = div_up(k->W, wo);
    const int sh = eff_seg(k);
    if (part && part->a1 > 0) {
        *segs = div_up(part->a1 - part->a0, sh) +
                (part->b1 > part->b0 ? div_up(part->b1 - part->b0, sh) : 0);
        pad = false;
    } else {
        *segs = div_up(k->H, sh);
    }
    const int tasks = *strips * *segs;
    *blocks = div_up(tasks, k->warps);
    if (k->resident_blocks > 0) *blocks = std::min(*blocks, k->resident_blocks);
    if (part && part->blocks > 0) *blocks = std::min(*blocks, part->blocks);
    if (use_walk2(k)) {
        // per warp: a ring of 6 rows, the vertical pair coefficients and one
        // mbarrier per ring slot (of 1 or 2 rows)
        *smem = (size_t)k->warps * (walk_window(k) * slot_bytes(k->C, k->fp32, k->imag,
                                                                (k->phase & 3) == 3) +
                                    tsb::w2_vlen(eff_seg(k), k->rot) * 2 * (k->fp32 ? 4 : 8) +
                                    (walk_window(k) / walk_rows(k)) * 8);
        if (k->overlap && pad) {
            // with programmatic dependent launch the next step's blocks are
            // placed as soon as an SM has room: reserve enough shared memory
            // that no SM holds more blocks of this step and the next together
            // than the grid's share per SM, so every SM receives the same
            // share of the next step
            const int per_sm = div_up(div_up((long)tasks, k->warps), k->num_sms);
            const size_t floor_b = (size_t)kSmemPerSm / (per_sm + 1) - kSmemReservedPerBlock + 128;
            *smem = std::max(*smem, floor_b);
        }
        return;
    }
    // per warp: ring slots + one mbarrier per ring slot
    *smem = (size_t)k->warps *
            (k->ring * slot_bytes(k->C, k->fp32, k->imag, k->phase == 3 || k->phase == 7) +
             8 * k->ring);
}

// xr1 > xr0: the rows whose x halo is refreshed (default: the reference's
// [inner_y0, inner_y0 + dim_y - 2 halo_y)).
template <typename T>
int launch_halo_t(ts_b200_kernel *k, cudaStream_t stream = nullptr, int xr0 = 0, int xr1 = 0) {
    if (!stream) stream = k->stream;
    if (xr1 <= xr0) {
        xr0 = k->d.inner_y0;
        xr1 = k->d.inner_y0 + k->H - 2 * k->d.halo_y;
    }
    if (!(k->d.periodic_x || k->d.periodic_y)) return TS_B200_OK;
    const int hx = k->d.halo_x, hy = k->d.halo_y;
    const int nx = k->d.periodic_x ? 2 * hx * k->H : 0;
    const int ny = k->d.periodic_y ? 2 * hy * (k->d.periodic_x ? k->W - 2 * hx : k->W) : 0;
    const int n = nx + ny;
    if (n <= 0) return TS_B200_OK;
    const int threads = 256;
    const int nb = std::min(div_up(n, threads), 4096);
    halo_kernel<T><<<nb, threads, 0, stream>>>(reinterpret_cast<Cx<T> *>(k->psi[k->cur]), k->W,
                                                  k->H, k->P, hx, hy, k->d.periodic_x,
                                                  k->d.periodic_y, xr0, xr1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(k, e, "halo kernel launch");
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

}  // namespace

template <typename T>
void tsbh::fill_step_constants(const ts_b200_kernel *k, StepArgs<T> &a) {
    a.pot = k->tab;
    a.row_ab = k->row_ab;
    a.col_ab = k->col_ab;
    a.W = k->W;
    a.H = k->H;
    a.P = k->P;
    a.ix0 = k->d.inner_x0;
    a.ix1 = k->d.inner_x1;
    a.iy0 = k->d.inner_y0;
    a.iy1 = k->d.inner_y1;
    a.aH = (T)k->d.a_h;
    a.bH = (T)k->d.b_h;
    a.aV = (T)k->d.a_v;
    a.bV = (T)k->d.b_v;
    if (sizeof(T) == 4) {
        // delta form: a - 1 from the angle, without cancellation
        const double kx = k->imag ? asinh(k->d.b_h) : asin(k->d.b_h);
        const double ky = k->imag ? asinh(k->d.b_v) : asin(k->d.b_v);
        const double amh = k->imag ? cosh_m1(kx) : cos_m1(kx);
        const double amv = k->imag ? cosh_m1(ky) : cos_m1(ky);
        float fa, fb;
        if (k->imag) {
            a.aH = (T)amh;
            a.aV = (T)amv;
        } else {
            unimodular_float_pair(amh, k->d.b_h, 16, &fa, &fb);
            a.aH = (T)fa;
            a.bH = (T)fb;
            unimodular_float_pair(amv, k->d.b_v, 16, &fa, &fb);
            a.aV = (T)fa;
            a.bV = (T)fb;
        }
    }
    a.ca = (T)k->d.coupling;
    a.caa = (T)k->d.lhy_coupling;
    a.scal = k->scal;
    a.kin_sched = k->kin_sched;
    a.sched_len = kSchedLen;
    a.dxdy = k->d.delta_x * k->d.delta_y;
    a.norm0 = k->d.norm0;
    a.pb = k->pb;
    a.pb_scale = k->pb_scale;
    a.cab = (T)k->cab;
    a.rabi_cc = (T)k->rabi[0];
    a.rabi_sr = (T)k->rabi[1];
    a.rabi_si = (T)k->rabi[2];
    a.rabi_or = (T)k->rabi[3];
    a.rabi_oi = (T)k->rabi[4];
    a.rad = k->rad;
    a.mirror_sign = (T)(k->d.angular_momentum % 2 == 0 ? 1 : -1);
}
template void tsbh::fill_step_constants<double>(const ts_b200_kernel *, StepArgs<double> &);
template void tsbh::fill_step_constants<float>(const ts_b200_kernel *, StepArgs<float> &);

namespace {

// Resident blocks of this variant and shape (the persistent grid size) and,
// from them, the segment height.
template <typename T>
int configure_t(ts_b200_kernel *k) {
    if (k->resident_blocks > 0) return TS_B200_OK;
    int strips, segs, blocks;
    size_t smem;
    geometry(k, &strips, &segs, &blocks, &smem, false);
    StepArgs<T> a0{};
    int bps = 0;
    cudaError_t e = dispatch_step<T>(k->C, k->imag, k->rot, k->phase, walk_rows(k), a0, k->warps,
                                     smem, 0, k->stream, &bps);
    if (e != cudaSuccess) return cuda_fail(k, e, "step kernel configuration");
    if (bps < 1) return fail(k, TS_B200_UNSUPPORTED, "step kernel does not fit on an SM");
    k->resident_blocks = bps * k->num_sms;
    if (k->auto_seg) auto_segments(k);
    return TS_B200_OK;
}

// One fused step from buffer `in` to buffer `out` (no buffer flip, no halo);
// dry: configure and size the scratch only.
template <typename T>
int launch_step_buffers_t(ts_b200_kernel *k, const void *in, void *out, bool dry) {
    int strips, segs, blocks;
    size_t smem;
    const int c = configure_t<T>(k);
    if (c) return c;
    geometry(k, &strips, &segs, &blocks, &smem);
    const size_t nwarps = (size_t)std::max(blocks, 1) * k->warps;
    if (k->imag && nwarps > k->partials_cap) {
        if (k->partials) cudaFree(k->partials);
        k->partials = nullptr;
        TSB_CHECK(k, cudaMalloc(&k->partials, nwarps * sizeof(double)));
        k->partials_cap = nwarps;
    }
    if (dry) blocks = 0;
    StepArgs<T> a{};
    a.psi_in = in;
    a.psi_out = out;
    tsbh::fill_step_constants(k, a);
    a.n_strips = strips;
    a.n_segs = segs;
    a.seg_h = eff_seg(k);
    a.ring = use_walk2(k) ? walk_window(k) / walk_rows(k) : k->ring;
    a.partials = k->partials;
    int phase = k->phase;
    if (k->vpot) {
        // the table made in the step from the potential rows
        a.pot = k->vpot;
        a.pot_pitch = k->vpot_pitch;
        a.pot_dt = k->vpot_dt;
        phase |= 16;
    }
    cudaError_t e = dispatch_step<T>(k->C, k->imag, k->rot, phase, walk_rows(k), a, k->warps,
                                     smem, blocks, k->stream, nullptr, k->overlap);
    if (e != cudaSuccess) return cuda_fail(k, e, "step kernel launch");
    if (!dry) g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

template <typename T>
int launch_step_t(ts_b200_kernel *k, int exchange, bool dry = false) {
    const int s = launch_step_buffers_t<T>(k, k->psi[k->cur], k->psi[1 - k->cur], dry);
    if (s || dry) return s;
    k->cur = 1 - k->cur;
    if (exchange) {
        const int st = launch_halo_t<T>(k);
        if (st) return st;
    }
    return TS_B200_OK;
}

int launch_step(ts_b200_kernel *k, int exchange, bool dry = false) {
    return k->fp32 ? launch_step_t<float>(k, exchange, dry) : launch_step_t<double>(k, exchange, dry);
}

template <typename T>
int launch_step_part_t(ts_b200_kernel *k, const void *in, void *out, const tsbh::StepPart &p) {
    const int c = configure_t<T>(k);
    if (c) return c;
    if (p.a1 > 0 && (p.a0 < 0 || p.a1 <= p.a0 || p.a1 > k->H || (p.a0 & 1) ||
                     (p.b1 > p.b0 && (p.b0 < 0 || p.b1 > k->H || (p.b0 & 1)))))
        return fail(k, TS_B200_INVALID_ARGUMENT, "step part: row windows");
    const bool pdl = p.pdl && p.a1 == 0 && k->overlap && use_walk2(k);
    int strips, segs, blocks;
    size_t smem;
    geometry(k, &strips, &segs, &blocks, &smem, pdl, &p);
    double *partials = p.partials;
    if (k->imag && !partials) {
        const size_t nb = (size_t)std::max(blocks, 1);
        if (nb * k->warps > k->partials_cap) {
            if (k->partials) cudaFree(k->partials);
            k->partials = nullptr;
            k->partials_cap = 0;
            TSB_CHECK(k, cudaMalloc(&k->partials, nb * k->warps * sizeof(double)));
            k->partials_cap = nb * k->warps;
        }
        partials = k->partials;
    }
    StepArgs<T> a{};
    a.psi_in = in;
    a.psi_out = out;
    tsbh::fill_step_constants(k, a);
    a.n_strips = strips;
    a.n_segs = segs;
    a.seg_h = eff_seg(k);
    a.ring = use_walk2(k) ? walk_window(k) / walk_rows(k) : k->ring;
    a.partials = partials;
    a.inv_copy = p.inv_copy;
    if (p.a1 > 0) {
        a.win_n0 = div_up(p.a1 - p.a0, a.seg_h);
        a.win_a0 = p.a0;
        a.win_a1 = p.a1;
        a.win_b0 = p.b0;
        a.win_b1 = p.b1 > p.b0 ? p.b1 : p.b0;
    }
    a.ticket = p.ticket;
    a.pair_norm = p.pair_norm;
    a.pair_ticket = p.pair_ticket;
    a.pair_slot = p.pair_slot;
    cudaError_t e = dispatch_step<T>(k->C, k->imag, k->rot, k->phase, walk_rows(k), a, k->warps,
                                     smem, blocks, p.stream ? p.stream : k->stream, nullptr, pdl);
    if (e != cudaSuccess) return cuda_fail(k, e, "step part launch");
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

}  // namespace

int tsbh::configure_step(ts_b200_kernel *k) {
    return k->fp32 ? configure_t<float>(k) : configure_t<double>(k);
}

int tsbh::part_blocks(const ts_b200_kernel *k, const tsbh::StepPart &p) {
    int strips, segs, blocks;
    size_t smem;
    geometry(k, &strips, &segs, &blocks, &smem, false, &p);
    return std::max(blocks, 1);
}

int tsbh::launch_step_part(ts_b200_kernel *k, const void *in, void *out, const tsbh::StepPart &p) {
    return k->fp32 ? launch_step_part_t<float>(k, in, out, p)
                   : launch_step_part_t<double>(k, in, out, p);
}

int tsbh::step_reach_rows(const ts_b200_kernel *k) { return k->rot ? 6 : 4; }  // Variant::HY

int tsbh::launch_halo_on(ts_b200_kernel *k, cudaStream_t stream, int xr0, int xr1) {
    return k->fp32 ? launch_halo_t<float>(k, stream, xr0, xr1)
                   : launch_halo_t<double>(k, stream, xr0, xr1);
}

int tsbh::launch_step_tile(ts_b200_kernel *k, int exchange) { return launch_step(k, exchange); }

int tsbh::set_norm0(ts_b200_kernel *k, double norm0) {
    if (!k->imag || !(norm0 > 0.0)) return fail(k, TS_B200_INVALID_ARGUMENT, "norm0");
    if (k->d.norm0 != norm0) {
        k->d.norm0 = norm0;
        drop_graph(k);
    }
    return TS_B200_OK;
}

int tsbh::launch_step_buffers(ts_b200_kernel *k, const void *in, void *out) {
    return k->fp32 ? launch_step_buffers_t<float>(k, in, out, false)
                   : launch_step_buffers_t<double>(k, in, out, false);
}

namespace {

int kernels_per_step(const ts_b200_kernel *k, int exchange) {
    return 1 + ((exchange && (k->d.periodic_x || k->d.periodic_y)) ? 1 : 0);
}

int check_device_error(ts_b200_kernel *k) {
    int err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, &k->scal->error, sizeof(int), cudaMemcpyDeviceToHost,
                                    k->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(k->stream);
    if (e != cudaSuccess) return cuda_fail(k, e, "device status read");
    if (err) {
        int zero = 0;
        cudaMemcpy(&k->scal->error, &zero, sizeof(int), cudaMemcpyHostToDevice);
        return fail(k, TS_B200_DEVICE_TIMEOUT,
                    "a bounded wait in the step kernel gave up (row copy did not complete)");
    }
    return TS_B200_OK;
}

void fill_red_args(ts_b200_kernel *k, RedArgs &a) {
    a.psi = k->psi[k->cur];
    a.W = k->W;
    a.H = k->H;
    a.P = k->P;
    a.ix0 = k->d.inner_x0;
    a.ix1 = k->d.inner_x1;
    a.iy0 = k->d.inner_y0;
    a.iy1 = k->d.inner_y1;
    a.scal = k->scal;
    a.use_scale = k->imag ? 1 : 0;
    a.dx = k->d.delta_x;
    a.dy = k->d.delta_y;
    a.partials = k->red_partials;
    a.out = k->red_out;
    a.ticket = k->red_ticket;
    a.cyl = k->cyl ? 1 : 0;
}

int red_blocks(const ts_b200_kernel *k) {
    const long n = (long)(k->d.inner_x1 - k->d.inner_x0) * (k->d.inner_y1 - k->d.inner_y0);
    return std::max(1, std::min(RED_MAX_BLOCKS, div_up(n, RED_THREADS)));
}

int read_red(ts_b200_kernel *k, double *host, int nterms) {
    TSB_CHECK(k, cudaMemcpyAsync(host, k->red_out, nterms * sizeof(double), cudaMemcpyDeviceToHost,
                                 k->stream));
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    return TS_B200_OK;
}

// Radial pair coefficients per tile column x (the pair (x, x+1); the tile
// starts at the axis), computed on the host with the C library as
// src/cpucylindrical.cpp:11-35 (real time) and :50-74 (imaginary time) do,
// including their choice of circular functions for the first pair in real time
// and hyperbolic ones past it (and the other way round in imaginary time).
// Stored as (a, b), (c, 0); a - 1 in float (delta form).
template <typename T>
int upload_radial(ts_b200_kernel *k) {
    const int W = k->W;
    Cx<T> *tab = new (std::nothrow) Cx<T>[2 * (size_t)W];
    if (!tab) return fail(k, TS_B200_OUT_OF_MEMORY, "host allocation for the radial table");
    const double kin = k->d.kin_radial;
    for (int x = 0; x < W; ++x) {
        double a, am1, b, c;
        if (x == 0) {
            const double kr = 2 * kin;
            a = k->imag ? std::cosh(kr) : std::cos(kr);
            am1 = k->imag ? cosh_m1(kr) : cos_m1(kr);
            b = c = k->imag ? -std::sinh(kr) : -std::sin(kr);
        } else {
            const double xd = (double)x;
            const double kr = kin / std::sqrt(xd * xd - 0.25);
            const double ratio = std::sqrt((2 * xd + 1) / (2 * xd - 1));
            const double sk = k->imag ? std::sin(kr) : std::sinh(kr);
            a = k->imag ? std::cos(kr) : std::cosh(kr);
            am1 = k->imag ? cos_m1(kr) : cosh_m1(kr);
            b = sk * ratio;
            c = -sk / ratio;
        }
        tab[2 * x] = Cx<T>{(T)(sizeof(T) == 4 ? am1 : a), (T)b};
        tab[2 * x + 1] = Cx<T>{(T)c, T(0)};
    }
    cudaError_t e = cudaMemcpy(k->rad, tab, sizeof(Cx<T>) * 2 * (size_t)W, cudaMemcpyHostToDevice);
    delete[] tab;
    if (e != cudaSuccess) return cuda_fail(k, e, "radial table upload");
    return TS_B200_OK;
}

// Rotation coefficients per row and column, computed on the host with the
// C library exactly as src/cpucartesian.cpp:146-147,165-166 does.
template <typename T>
int upload_rotation(ts_b200_kernel *k) {
    const int W = k->W, H = k->H;
    Cx<T> *rows = new (std::nothrow) Cx<T>[H];
    Cx<T> *cols = new (std::nothrow) Cx<T>[W];
    if (!rows || !cols) {
        delete[] rows;
        delete[] cols;
        return fail(k, TS_B200_OUT_OF_MEMORY, "host allocation for rotation tables");
    }
    const int offx = (int)k->d.rot_offset_x, offy = (int)k->d.rot_offset_y;
    for (int y = 0; y < H; ++y) {
        const double ang = -0.5 * k->d.alpha_y * (y + offy);
        const double a = k->imag ? std::cosh(ang) : std::cos(ang);
        const double b = k->imag ? std::sinh(ang) : std::sin(ang);
        if (sizeof(T) == 4) {
            const double am1 = k->imag ? cosh_m1(ang) : cos_m1(ang);
            float fa = (float)am1, fb = (float)b;
            if (!k->imag) unimodular_float_pair(am1, b, 16, &fa, &fb);
            rows[y] = Cx<T>{(T)fa, (T)fb};
        } else {
            rows[y] = Cx<T>{(T)a, (T)b};
        }
    }
    for (int x = 0; x < W; ++x) {
        const double ang = k->d.alpha_x * (x + offx);
        const double a = k->imag ? std::cosh(ang) : std::cos(ang);
        const double b = k->imag ? std::sinh(ang) : std::sin(ang);
        if (sizeof(T) == 4) {
            const double am1 = k->imag ? cosh_m1(ang) : cos_m1(ang);
            float fa = (float)am1, fb = (float)b;
            if (!k->imag) unimodular_float_pair(am1, b, 16, &fa, &fb);
            cols[x] = Cx<T>{(T)fa, (T)fb};
        } else {
            cols[x] = Cx<T>{(T)a, (T)b};
        }
    }
    cudaError_t e = cudaMemcpy(k->row_ab, rows, sizeof(Cx<T>) * H, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(k->col_ab, cols, sizeof(Cx<T>) * W, cudaMemcpyHostToDevice);
    delete[] rows;
    delete[] cols;
    if (e != cudaSuccess) return cuda_fail(k, e, "rotation table upload");
    return TS_B200_OK;
}

// FP32 real time: kinetic coefficients per step in delta form, each the
// float nearest to the exact value plus the error carried from the previous
// entries (first-order sigma-delta), so that any run of consecutive entries
// sums to the exact total within half an ulp.
int upload_kinetic_schedule(ts_b200_kernel *k) {
    const double kx = asin(k->d.b_h), ky = asin(k->d.b_v);
    const double exact[4] = {cos_m1(kx), k->d.b_h, cos_m1(ky), k->d.b_v};
    double carry[4] = {0.0, 0.0, 0.0, 0.0};
    float4 *host = new (std::nothrow) float4[kSchedLen];
    if (!host) return fail(k, TS_B200_OUT_OF_MEMORY, "host allocation for the kinetic schedule");
    for (int i = 0; i < kSchedLen; ++i) {
        float c[4];
        for (int j = 0; j < 4; ++j) {
            c[j] = (float)(exact[j] + carry[j]);
            carry[j] += exact[j] - (double)c[j];
        }
        host[i] = make_float4(c[0], c[1], c[2], c[3]);
    }
    cudaError_t e = cudaMemcpy(k->kin_sched, host, (size_t)kSchedLen * sizeof(float4),
                               cudaMemcpyHostToDevice);
    delete[] host;
    if (e != cudaSuccess) return cuda_fail(k, e, "kinetic schedule upload");
    return TS_B200_OK;
}

int grid_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 8192)); }

// The pending factor from a norm summed over several tiles (one lattice
// split across ranks): src/cpukernel.cpp:537-562 with the MPI_Allgather sum.
__global__ void renorm_from_kernel(Scalars *scal, const double *total, double norm0) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && scal->renorm)
        scal->pending_inv = 1.0 / sqrt(*total / norm0);
}

// A tile that is one species of a pair steps only through the pair.
int reject_pair_mode(ts_b200_kernel *k) {
    return fail(k, TS_B200_UNSUPPORTED, "the tile is one component of a pair: step the pair");
}

}  // namespace

// ================================================================ C ABI
extern "C" {

const char *ts_b200_version(void) { return "ts_b200 1.0 (sm_100a)"; }

uint64_t ts_b200_launch_count(void) { return g_launches.load(); }

const char *ts_b200_status_string(int s) {
    switch (s) {
        case TS_B200_OK: return "ok";
        case TS_B200_INVALID_ARGUMENT: return "invalid argument";
        case TS_B200_CUDA_ERROR: return "CUDA error";
        case TS_B200_OUT_OF_MEMORY: return "out of device memory";
        case TS_B200_UNSUPPORTED: return "unsupported configuration";
        case TS_B200_DEVICE_TIMEOUT: return "device wait timed out";
        case TS_B200_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char *ts_b200_last_error(const ts_b200_kernel *k) { return k ? k->err.c_str() : ""; }

int ts_b200_create(const ts_b200_desc *d, ts_b200_kernel **out) {
    if (!d || !out) return TS_B200_INVALID_ARGUMENT;
    *out = nullptr;
    if (d->dim_x < 1 || d->dim_y < 1 || d->inner_x0 < 0 || d->inner_x1 > d->dim_x ||
        d->inner_x0 >= d->inner_x1 || d->inner_y0 < 0 || d->inner_y1 > d->dim_y ||
        d->inner_y0 >= d->inner_y1 || d->halo_x < 0 || d->halo_y < 0 ||
        (d->precision != TS_B200_FP64 && d->precision != TS_B200_FP32))
        return TS_B200_INVALID_ARGUMENT;
    if ((long)d->dim_x * d->dim_y > (1L << 31) - 1) return TS_B200_UNSUPPORTED;
    if (d->periodic_x && d->dim_x < 2 * d->halo_x) return TS_B200_INVALID_ARGUMENT;
    if (d->periodic_y && d->dim_y < 2 * d->halo_y) return TS_B200_INVALID_ARGUMENT;
    // cylindrical: the radial axis is not periodic, and the rotating frame is
    // not combined with it here
    if (d->cylindrical && (d->periodic_x || (d->alpha_x != 0.0 && d->alpha_y != 0.0)))
        return TS_B200_UNSUPPORTED;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return TS_B200_NO_DEVICE;
    ts_b200_kernel *k = new (std::nothrow) ts_b200_kernel();
    if (!k) return TS_B200_OUT_OF_MEMORY;
    k->d = *d;
    k->W = d->dim_x;
    k->H = d->dim_y;
    k->P = (d->dim_x + 3) & ~3;
    k->fp32 = d->precision == TS_B200_FP32;
    k->imag = d->imag_time != 0;
    k->rot = d->alpha_x != 0.0 && d->alpha_y != 0.0;
    k->phase = d->lhy_coupling != 0.0 ? 2 : (d->coupling != 0.0 ? 1 : 0);
    k->cyl = d->cylindrical != 0;
    if (k->cyl) k->phase |= 4;
    k->cell = k->fp32 ? 8 : 16;
    k->tab_cell = k->imag ? k->cell / 2 : k->cell;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&k->num_sms, cudaDevAttrMultiProcessorCount, dev);
    k->device = dev;
    choose_launch(k);
    const size_t ncell = (size_t)k->P * k->H;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    alloc(&k->psi[0], ncell * k->cell);
    alloc(&k->psi[1], ncell * k->cell);
    alloc(&k->tab, ncell * k->tab_cell);
    alloc((void **)&k->scal, sizeof(Scalars));
    alloc((void **)&k->staging, (size_t)2 * k->W * k->H * sizeof(double));
    alloc((void **)&k->red_partials, (size_t)RED_MAX_BLOCKS * RED_MAX_TERMS * sizeof(double));
    alloc((void **)&k->red_out, RED_MAX_TERMS * sizeof(double));
    alloc((void **)&k->red_ticket, sizeof(unsigned int));
    if (k->rot) {
        alloc(&k->row_ab, (size_t)k->H * (k->fp32 ? 8 : 16));
        alloc(&k->col_ab, (size_t)k->W * (k->fp32 ? 8 : 16));
    }
    if (k->fp32 && !k->imag) alloc((void **)&k->kin_sched, (size_t)kSchedLen * sizeof(float4));
    if (k->cyl) alloc(&k->rad, (size_t)k->W * 2 * k->cell);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&k->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        int s = cuda_fail(nullptr, e, "allocation");
        ts_b200_destroy(k);
        return s;
    }
    k->stream = k->own_stream;
    Scalars s0{};
    s0.pending_inv = 1.0;
    s0.prev_inv = 1.0;
    s0.norm_target = d->norm0;
    s0.renorm = (k->imag && d->norm0 != 0.0) ? 1 : 0;
    e = cudaMemcpy(k->scal, &s0, sizeof s0, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        int s = cuda_fail(nullptr, e, "scalar init");
        ts_b200_destroy(k);
        return s;
    }
    if (k->rot) {
        int s = k->fp32 ? upload_rotation<float>(k) : upload_rotation<double>(k);
        if (s != TS_B200_OK) {
            ts_b200_destroy(k);
            return s;
        }
    }
    if (k->cyl) {
        int s = k->fp32 ? upload_radial<float>(k) : upload_radial<double>(k);
        if (s != TS_B200_OK) {
            ts_b200_destroy(k);
            return s;
        }
    }
    if (k->kin_sched) {
        int s = upload_kinetic_schedule(k);
        if (s != TS_B200_OK) {
            ts_b200_destroy(k);
            return s;
        }
    }
    *out = k;
    return TS_B200_OK;
}

int ts_b200_destroy(ts_b200_kernel *k) {
    if (!k) return TS_B200_OK;
    drop_graph(k);
    if (k->own_stream) cudaStreamSynchronize(k->own_stream);
    if (k->stream && k->stream != k->own_stream) cudaStreamSynchronize(k->stream);
    void *bufs[] = {k->psi[0], k->psi[1], k->tab, k->row_ab, k->col_ab, k->partials, k->scal,
                    k->staging, k->vtab, k->red_partials, k->red_out, k->red_ticket,
                    k->kin_sched, k->rad};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (k->own_stream) cudaStreamDestroy(k->own_stream);
    if (k->ev_order) cudaEventDestroy(k->ev_order);
    delete k;
    return TS_B200_OK;
}

int ts_b200_set_stream(ts_b200_kernel *k, void *stream) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    drop_graph(k);
    k->stream = stream ? reinterpret_cast<cudaStream_t>(stream) : k->own_stream;
    return TS_B200_OK;
}

namespace {
int order_streams(ts_b200_kernel *k, cudaStream_t first, cudaStream_t then) {
    if (first == then) return TS_B200_OK;
    if (!k->ev_order) TSB_CHECK(k, cudaEventCreateWithFlags(&k->ev_order, cudaEventDisableTiming));
    TSB_CHECK(k, cudaEventRecord(k->ev_order, first));
    TSB_CHECK(k, cudaStreamWaitEvent(then, k->ev_order, 0));
    return TS_B200_OK;
}
}  // namespace

int ts_b200_stream_wait(ts_b200_kernel *k, void *stream) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    return order_streams(k, reinterpret_cast<cudaStream_t>(stream), k->stream);
}

int ts_b200_stream_signal(ts_b200_kernel *k, void *stream) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    return order_streams(k, k->stream, reinterpret_cast<cudaStream_t>(stream));
}

int ts_b200_synchronize(ts_b200_kernel *k) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    return check_device_error(k);
}

int ts_b200_set_state(ts_b200_kernel *k, const double *re, const double *im, size_t stride) {
    if (!k || !re || !im || stride < (size_t)k->W) return TS_B200_INVALID_ARGUMENT;
    double *sre = k->staging, *sim = k->staging + (size_t)k->W * k->H;
    TSB_CHECK(k, cudaMemcpy2DAsync(sre, k->W * sizeof(double), re, stride * sizeof(double),
                                   k->W * sizeof(double), k->H, cudaMemcpyHostToDevice, k->stream));
    TSB_CHECK(k, cudaMemcpy2DAsync(sim, k->W * sizeof(double), im, stride * sizeof(double),
                                   k->W * sizeof(double), k->H, cudaMemcpyHostToDevice, k->stream));
    const size_t n = (size_t)k->P * k->H;
    if (k->fp32)
        pack_state_kernel<float><<<grid_for(n), 256, 0, k->stream>>>(
            reinterpret_cast<Cx<float> *>(k->psi[k->cur]), k->W, k->H, k->P, sre, sim, k->W);
    else
        pack_state_kernel<double><<<grid_for(n), 256, 0, k->stream>>>(
            reinterpret_cast<Cx<double> *>(k->psi[k->cur]), k->W, k->H, k->P, sre, sim, k->W);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    // a freshly uploaded state carries no pending renormalisation
    const double one = 1.0;
    TSB_CHECK(k, cudaMemcpyAsync(&k->scal->pending_inv, &one, sizeof(double), cudaMemcpyHostToDevice,
                                 k->stream));
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    return TS_B200_OK;
}

int ts_b200_set_exp_potential(ts_b200_kernel *k, const double *re, const double *im,
                              size_t stride) {
    if (!k || !re || (!im && !k->imag) || stride < (size_t)k->W) return TS_B200_INVALID_ARGUMENT;
    double *sre = k->staging, *sim = k->staging + (size_t)k->W * k->H;
    TSB_CHECK(k, cudaMemcpy2DAsync(sre, k->W * sizeof(double), re, stride * sizeof(double),
                                   k->W * sizeof(double), k->H, cudaMemcpyHostToDevice, k->stream));
    if (im)
        TSB_CHECK(k, cudaMemcpy2DAsync(sim, k->W * sizeof(double), im, stride * sizeof(double),
                                       k->W * sizeof(double), k->H, cudaMemcpyHostToDevice,
                                       k->stream));
    else
        TSB_CHECK(k, cudaMemsetAsync(sim, 0, (size_t)k->W * k->H * sizeof(double), k->stream));
    const size_t n = (size_t)k->P * k->H;
    if (k->fp32)
        pack_table_kernel<float><<<grid_for(n), 256, 0, k->stream>>>(k->tab, k->imag, k->W, k->H,
                                                                      k->P, sre, sim, k->W);
    else
        pack_table_kernel<double><<<grid_for(n), 256, 0, k->stream>>>(k->tab, k->imag, k->W, k->H,
                                                                       k->P, sre, sim, k->W);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    return TS_B200_OK;
}

int ts_b200_set_state_device(ts_b200_kernel *k, const void *aos, size_t pitch) {
    if (!k || !aos || pitch < (size_t)k->W) return TS_B200_INVALID_ARGUMENT;
    TSB_CHECK(k, cudaMemcpy2DAsync(k->psi[k->cur], k->P * k->cell, aos, pitch * k->cell,
                                   k->W * k->cell, k->H, cudaMemcpyDeviceToDevice, k->stream));
    const double one = 1.0;
    TSB_CHECK(k, cudaMemcpyAsync(&k->scal->pending_inv, &one, sizeof(double), cudaMemcpyHostToDevice,
                                 k->stream));
    return TS_B200_OK;
}

int ts_b200_get_state_device(ts_b200_kernel *k, void *aos, size_t pitch) {
    if (!k || !aos || pitch < (size_t)k->W) return TS_B200_INVALID_ARGUMENT;
    const size_t n = (size_t)k->W * k->H;
    if (k->fp32)
        copy_tile_kernel<float><<<grid_for(n), 256, 0, k->stream>>>(
            reinterpret_cast<Cx<float> *>(aos), pitch,
            reinterpret_cast<const Cx<float> *>(k->psi[k->cur]), k->P, k->W, k->H, k->scal,
            k->imag ? 1 : 0);
    else
        copy_tile_kernel<double><<<grid_for(n), 256, 0, k->stream>>>(
            reinterpret_cast<Cx<double> *>(aos), pitch,
            reinterpret_cast<const Cx<double> *>(k->psi[k->cur]), k->P, k->W, k->H, k->scal,
            k->imag ? 1 : 0);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

int ts_b200_set_exp_potential_device(ts_b200_kernel *k, const void *table, size_t pitch) {
    if (!k || !table || pitch < (size_t)k->W) return TS_B200_INVALID_ARGUMENT;
    TSB_CHECK(k, cudaMemcpy2DAsync(k->tab, k->P * k->tab_cell, table, pitch * k->tab_cell,
                                   k->W * k->tab_cell, k->H, cudaMemcpyDeviceToDevice, k->stream));
    return TS_B200_OK;
}

int ts_b200_set_potential_device(ts_b200_kernel *k, const double *potential, size_t pitch,
                                 double delta_t) {
    if (!k || !potential || pitch < (size_t)k->W || !(delta_t > 0.0))
        return TS_B200_INVALID_ARGUMENT;
    launch_table_from_potential(k, potential, pitch, delta_t);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

namespace {
// The step can read the potential rows directly: FP64 real time, one
// component, cartesian, no rotating frame, the look-ahead walk with two rows
// per iteration; and the rows' copies aligned to 16 bytes (even width and
// pitch, aligned planes).
bool fused_potential_ok(const ts_b200_kernel *k, const double *V, size_t pitch, size_t slab) {
    return !k->fp32 && !k->imag && !k->rot && !k->cyl && !k->pair_mode && k->phase <= 2 &&
           use_walk2(k) && walk_rows(k) == 2 && k->C == 2 && (k->W % 2) == 0 &&
           (pitch % 2) == 0 && (slab % 2) == 0 && (reinterpret_cast<uintptr_t>(V) % 16) == 0;
}
}  // namespace

int ts_b200_evolve_potentials(ts_b200_kernel *k, const double *potentials, size_t pitch,
                              size_t slab, int count, double delta_t, int exchange) {
    if (!k || !potentials || count < 0 || pitch < (size_t)k->W || slab < pitch * k->H ||
        !(delta_t > 0.0))
        return TS_B200_INVALID_ARGUMENT;
    if (k->pair_mode) return reject_pair_mode(k);
    // FP64 real-time cartesian steps on the look-ahead walk read the
    // potential rows and form the table's entries themselves (no table pass:
    // 8 B instead of 16 B per cell read, the table's 24 B per cell not moved);
    // the table of the last potential is then built once, for later steps
    // (so a single step keeps the table pass: the same traffic either way)
    if (count >= 2 && fused_potential_ok(k, potentials, pitch, slab)) {
        int s = TS_B200_OK;
        for (int i = 0; i < count && s == TS_B200_OK; ++i) {
            k->vpot = potentials + (size_t)i * slab;
            k->vpot_pitch = pitch * sizeof(double);
            k->vpot_dt = delta_t;
            s = launch_step(k, exchange);
        }
        k->vpot = nullptr;
        if (s) return s;
        if (count > 0) {
            launch_table_from_potential(k, potentials + (size_t)(count - 1) * slab, pitch, delta_t);
            TSB_CHECK(k, cudaGetLastError());
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
        return TS_B200_OK;
    }
    for (int i = 0; i < count; ++i) {
        launch_table_from_potential(k, potentials + (size_t)i * slab, pitch, delta_t);
        TSB_CHECK(k, cudaGetLastError());
        g_launches.fetch_add(1, std::memory_order_relaxed);
        const int s = launch_step(k, exchange);
        if (s) return s;
    }
    return TS_B200_OK;
}

int ts_b200_rows(ts_b200_kernel *k, int row0, int nrows, void **ptr, size_t *bytes) {
    if (!k || !ptr || !bytes || row0 < 0 || nrows < 0 || row0 + nrows > k->H)
        return TS_B200_INVALID_ARGUMENT;
    *ptr = static_cast<unsigned char *>(k->psi[k->cur]) + (size_t)row0 * k->P * k->cell;
    *bytes = (size_t)nrows * k->P * k->cell;
    return TS_B200_OK;
}

int ts_b200_last_norm(ts_b200_kernel *k, double **device_ptr) {
    if (!k || !device_ptr) return TS_B200_INVALID_ARGUMENT;
    *device_ptr = &k->scal->last_norm;
    return TS_B200_OK;
}

int ts_b200_renormalize_from(ts_b200_kernel *k, const double *total_norm) {
    if (!k || !total_norm) return TS_B200_INVALID_ARGUMENT;
    if (!k->imag) return TS_B200_OK;
    renorm_from_kernel<<<1, 32, 0, k->stream>>>(k->scal, total_norm, k->d.norm0);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

int ts_b200_step(ts_b200_kernel *k, int exchange) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    if (k->pair_mode) return reject_pair_mode(k);
    return launch_step(k, exchange);
}

int ts_b200_halo_exchange(ts_b200_kernel *k) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    return k->fp32 ? launch_halo_t<float>(k) : launch_halo_t<double>(k);
}

int ts_b200_evolve(ts_b200_kernel *k, int iterations) {
    if (!k || iterations < 0) return TS_B200_INVALID_ARGUMENT;
    if (k->pair_mode) return reject_pair_mode(k);
    if (iterations == 0) return TS_B200_OK;
    // Steps 0 .. iterations-2 refresh the halo; the last one does not
    // (src/solver.cpp:203-209).  Runs of G exchanging steps starting from
    // buffer 0 are replayed from one CUDA graph (G even, so the graph leaves
    // the buffers as it found them).
    const int G = 32;
    int remaining = iterations - 1;  // exchanging steps
    if (remaining > 0 && k->cur != 0) {
        int s = launch_step(k, 1);
        if (s) return s;
        --remaining;
    }
    if (remaining >= G) {
        if (!k->graph || k->graph_steps != G) {
            drop_graph(k);
            int s0 = launch_step(k, 1, true);  // scratch and attributes before capture
            if (s0) return s0;
            cudaGraph_t g = nullptr;
            TSB_CHECK(k, cudaStreamBeginCapture(k->stream, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = g_launches.load();
            int s = TS_B200_OK;
            for (int i = 0; i < G && s == TS_B200_OK; ++i) s = launch_step(k, 1);
            cudaError_t e = cudaStreamEndCapture(k->stream, &g);
            g_launches.store(before);  // captured launches are counted when replayed
            if (s != TS_B200_OK || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                (void)cudaGetLastError();  // do not leave the capture error to later calls
                if (s != TS_B200_OK) return s;
            }
            if (e != cudaSuccess) return cuda_fail(k, e, "graph capture");
            e = cudaGraphInstantiate(&k->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(k, e, "graph instantiate");
            k->graph_steps = G;
        }
        const int per = kernels_per_step(k, 1);
        while (remaining >= G) {
            TSB_CHECK(k, cudaGraphLaunch(k->graph, k->stream));
            g_launches.fetch_add((uint64_t)G * per, std::memory_order_relaxed);
            remaining -= G;
        }
    }
    for (; remaining > 0; --remaining) {
        int s = launch_step(k, 1);
        if (s) return s;
    }
    return launch_step(k, 0);
}

int ts_b200_get_sample(ts_b200_kernel *k, size_t dest_stride, size_t x, size_t y, size_t width,
                       size_t height, double *re, double *im) {
    if (!k || !re || !im || x + width > (size_t)k->W || y + height > (size_t)k->H ||
        dest_stride < width)
        return TS_B200_INVALID_ARGUMENT;
    if (width == 0 || height == 0) return TS_B200_OK;
    double *sre = k->staging, *sim = k->staging + width * height;
    const size_t n = width * height;
    if (k->fp32)
        unpack_state_kernel<float><<<grid_for(n), 256, 0, k->stream>>>(
            reinterpret_cast<const Cx<float> *>(k->psi[k->cur]), k->P, (int)x, (int)y, (int)width,
            (int)height, k->scal, k->imag ? 1 : 0, sre, sim);
    else
        unpack_state_kernel<double><<<grid_for(n), 256, 0, k->stream>>>(
            reinterpret_cast<const Cx<double> *>(k->psi[k->cur]), k->P, (int)x, (int)y,
            (int)width, (int)height, k->scal, k->imag ? 1 : 0, sre, sim);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    TSB_CHECK(k, cudaMemcpy2DAsync(re, dest_stride * sizeof(double), sre, width * sizeof(double),
                                   width * sizeof(double), height, cudaMemcpyDeviceToHost,
                                   k->stream));
    TSB_CHECK(k, cudaMemcpy2DAsync(im, dest_stride * sizeof(double), sim, width * sizeof(double),
                                   width * sizeof(double), height, cudaMemcpyDeviceToHost,
                                   k->stream));
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    return check_device_error(k);
}

int ts_b200_squared_norm(ts_b200_kernel *k, double *out) {
    if (!k || !out) return TS_B200_INVALID_ARGUMENT;
    RedArgs a{};
    fill_red_args(k, a);
    const int nb = red_blocks(k);
    if (k->fp32) norm_kernel<float><<<nb, RED_THREADS, 0, k->stream>>>(a);
    else norm_kernel<double><<<nb, RED_THREADS, 0, k->stream>>>(a);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    double s = 0;
    int st = read_red(k, &s, 1);
    if (st) return st;
    *out = s * k->d.delta_x * k->d.delta_y;
    return TS_B200_OK;
}

int ts_b200_energies(ts_b200_kernel *k, const double *potential, const ts_b200_energy_params *p,
                     ts_b200_energy_result *out) {
    if (!k || !p || !out) return TS_B200_INVALID_ARGUMENT;
    if (potential) {
        if (!k->vtab) TSB_CHECK(k, cudaMalloc((void **)&k->vtab, (size_t)k->W * k->H * sizeof(double)));
        TSB_CHECK(k, cudaMemcpyAsync(k->vtab, potential, (size_t)k->W * k->H * sizeof(double),
                                     cudaMemcpyHostToDevice, k->stream));
        k->have_v = true;
    }
    if (!k->have_v) return fail(k, TS_B200_INVALID_ARGUMENT, "no potential uploaded for energies");
    RedArgs a{};
    fill_red_args(k, a);
    a.V = k->vtab;
    a.start_x = p->start_x;
    a.start_y = p->start_y;
    a.gnx = p->global_no_halo_dim_x;
    a.gny = p->global_no_halo_dim_y;
    a.Lx = p->length_x;
    a.Ly = p->length_y;
    a.mass = p->mass;
    a.g = p->coupling;
    a.glhy = p->lhy_coupling;
    a.omega = p->angular_velocity;
    const int nb = red_blocks(k);
    if (k->fp32) energy_kernel<float><<<nb, RED_THREADS, 0, k->stream>>>(a);
    else energy_kernel<double><<<nb, RED_THREADS, 0, k->stream>>>(a);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    double s[7];
    int st = read_red(k, s, 7);
    if (st) return st;
    // final arithmetic of src/solver.cpp:532-538,561
    out->kinetic = s[2] / s[1];
    out->rotational = s[4] / s[1];
    out->potential = s[3] / s[0];
    out->intra = s[5] / s[0];
    out->lhy = s[6] / s[0];
    out->total = out->kinetic + out->potential + out->intra + out->rotational + out->lhy;
    out->norm2 = s[0] * (k->d.delta_y * p->length_x /
                         (p->global_no_halo_dim_x - (k->cyl ? 1 : 0)));
    return TS_B200_OK;
}

int ts_b200_expectations(ts_b200_kernel *k, const ts_b200_energy_params *p,
                         ts_b200_expectation_result *out) {
    if (!k || !p || !out) return TS_B200_INVALID_ARGUMENT;
    RedArgs a{};
    fill_red_args(k, a);
    a.start_x = p->start_x;
    a.start_y = p->start_y;
    a.gnx = p->global_no_halo_dim_x;
    a.gny = p->global_no_halo_dim_y;
    a.Lx = p->length_x;
    a.Ly = p->length_y;
    const int nb = red_blocks(k);
    if (k->fp32) expect_kernel<float><<<nb, RED_THREADS, 0, k->stream>>>(a);
    else expect_kernel<double><<<nb, RED_THREADS, 0, k->stream>>>(a);
    TSB_CHECK(k, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    double s[10];
    int st = read_red(k, s, 10);
    if (st) return st;
    // final arithmetic of src/model.cpp:456-534
    const double ppx = -1. / k->d.delta_x, ppy = 1. / k->d.delta_y;
    out->mean_x = s[1] / s[0];
    out->mean_y = s[2] / s[0];
    out->mean_xx = s[3] / s[0];
    out->mean_yy = s[4] / s[0];
    out->mean_px = -s[5] * ppx / s[0];
    out->mean_py = -s[6] * ppy / s[0];
    out->mean_pxpx = -s[7] * ppx * ppx / s[0];
    out->mean_pypy = -s[8] * ppy * ppy / s[0];
    out->mean_lz = s[9] / s[0];
    out->norm2 = s[0] * (k->d.delta_x * k->d.delta_y);
    return TS_B200_OK;
}

int ts_b200_launch_info(const ts_b200_kernel *k, ts_b200_launch_shape *out) {
    if (!k || !out) return TS_B200_INVALID_ARGUMENT;
    int strips, segs, blocks;
    size_t smem;
    geometry(k, &strips, &segs, &blocks, &smem);
    out->cells_per_lane = k->C;
    out->segment_rows = eff_seg(k);
    out->warps_per_block = k->warps;
    out->ring_depth = use_walk2(k) ? walk_window(k) : k->ring;
    out->walk = walk_rows(k);
    out->strips = strips;
    out->segments = segs;
    out->blocks = blocks;
    out->threads = k->warps * 32;
    out->smem_bytes = (int64_t)smem;
    return TS_B200_OK;
}

int ts_b200_set_launch(ts_b200_kernel *k, int C, int seg_h, int warps, int ring) {
    if (!k) return TS_B200_INVALID_ARGUMENT;
    if (C != 0 && C != 2 && C != 4) return TS_B200_INVALID_ARGUMENT;
    if (C == 4 && k->rot && !(k->fp32 && k->walk2 > 0))
        return fail(k, TS_B200_UNSUPPORTED,
                    "rotation kernels use 2 cells per lane (4: single precision, look-ahead walk)");
    if (C == 4 && k->pair_mode) return fail(k, TS_B200_UNSUPPORTED, "pair kernels use 2 cells per lane");
    if (C == 4 && k->cyl) return fail(k, TS_B200_UNSUPPORTED, "cylindrical kernels use 2 cells per lane");
    if (warps != 0 && warps != 1 && warps != 2 && warps != 4 && warps != 8)
        return TS_B200_INVALID_ARGUMENT;
    if (warps == 8 && !use_walk2(k))
        return fail(k, TS_B200_UNSUPPORTED, "8 warps per block need the look-ahead walk");
    if (warps == 8 && k->rot)
        return fail(k, TS_B200_UNSUPPORTED, "rotating-frame kernels use blocks of at most 4 warps");
    if (ring != 0 && (ring < min_ring(k) || ring > 16))
        return fail(k, TS_B200_INVALID_ARGUMENT, "ring depth out of range for this variant");
    if (seg_h < 0) return TS_B200_INVALID_ARGUMENT;
    if (C) k->C = C;
    if (seg_h) {
        k->seg_h = seg_h;
        k->auto_seg = false;
    }
    if (warps) k->warps = warps;
    if (ring) k->ring = ring;
    k->resident_blocks = 0;
    int strips, segs, blocks;
    size_t smem;
    geometry(k, &strips, &segs, &blocks, &smem);
    if (smem > 227 * 1024) return fail(k, TS_B200_INVALID_ARGUMENT, "ring does not fit in shared memory");
    drop_graph(k);
    return TS_B200_OK;
}

int ts_b200_set_walk(ts_b200_kernel *k, int walk) {
    if (!k || walk < 0 || walk > 2) return TS_B200_INVALID_ARGUMENT;
    if (k->walk2 == walk) return TS_B200_OK;
    k->walk2 = walk;
    if (!use_walk2(k) && k->warps > 4) k->warps = 4;
    // the checked walk's rotating frame has 2 cells per lane
    if (walk == 0 && k->rot && k->C == 4) k->C = 2;
    k->resident_blocks = 0;
    drop_graph(k);
    return TS_B200_OK;
}

int ts_b200_set_overlap(ts_b200_kernel *k, int on) {
    if (!k || (on != 0 && on != 1)) return TS_B200_INVALID_ARGUMENT;
    if (k->overlap != (on == 1)) {
        k->overlap = on == 1;
        drop_graph(k);
    }
    return TS_B200_OK;
}

int ts_b200_autotune(ts_b200_kernel *k, int trial_steps) {
    if (!k || trial_steps < 1) return TS_B200_INVALID_ARGUMENT;
    if (k->pair_mode) return reject_pair_mode(k);
    // the trials step from the current buffer into the other one without
    // flipping, so the state is untouched; the scalars the step writes
    // (renormalisation, schedule step) are restored afterwards
    Scalars saved{};
    TSB_CHECK(k, cudaMemcpyAsync(&saved, k->scal, sizeof saved, cudaMemcpyDeviceToHost, k->stream));
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    const int C0 = k->C, seg0 = k->seg_h, warps0 = k->warps;
    const bool auto0 = k->auto_seg, overlap0 = k->overlap;
    cudaEvent_t e0, e1;
    TSB_CHECK(k, cudaEventCreate(&e0));
    TSB_CHECK(k, cudaEventCreate(&e1));
    float best_ms = -1.0f;
    int best_seg = seg0, best_warps = warps0;
    bool best_overlap = overlap0;
    int st = TS_B200_OK;
    // the look-ahead walk: blocks of 4 or 8 warps (4 or 2 in a rotating
    // frame), with and without programmatic dependent launch; the checked
    // walk: 4 or 2 warps
    const bool w2 = use_walk2(k);
    const int warp_opts[2] = {4, (w2 && !k->rot) ? 8 : 2};
    for (int trial = 0; trial < (w2 ? 4 : 2) && st == TS_B200_OK; ++trial) {
        const int warps = warp_opts[trial & 1];
        k->overlap = w2 ? ((trial >> 1) ? !overlap0 : overlap0) : overlap0;
        k->warps = warps;
        k->resident_blocks = 0;
        k->auto_seg = false;
        // resident blocks of this shape (the step kernel's occupancy)
        st = launch_step(k, 0, true);
        if (st) break;
        const int bps = std::max(1, k->resident_blocks / std::max(1, k->num_sms));
        // balanced shapes (one task per warp at b blocks per SM) and short
        // segments taken by the persistent warps in turn
        int cand[24], nc = 0;
        for (int b = 1; b <= bps && nc < 20; ++b) cand[nc++] = balanced_segments(k, b, warps);
        for (int sh : {32, 64, 128})
            if (sh < k->H) cand[nc++] = sh;
        for (int c = 0; c < nc && st == TS_B200_OK; ++c) {
            bool seen = false;
            for (int d = 0; d < c; ++d) seen = seen || cand[d] == cand[c];
            if (seen) continue;
            k->seg_h = cand[c];
            st = tsbh::launch_step_buffers(k, k->psi[k->cur], k->psi[1 - k->cur]);
            if (st) break;
            cudaEventRecord(e0, k->stream);
            for (int i = 0; i < trial_steps && st == TS_B200_OK; ++i)
                st = tsbh::launch_step_buffers(k, k->psi[k->cur], k->psi[1 - k->cur]);
            cudaEventRecord(e1, k->stream);
            cudaError_t e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                st = cuda_fail(k, e, "autotune timing");
                break;
            }
            if (best_ms < 0.0f || ms < best_ms) {
                best_ms = ms;
                best_seg = k->seg_h;
                best_warps = warps;
                best_overlap = k->overlap;
            }
        }
        if (st) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) {
        k->C = C0;
        k->seg_h = seg0;
        k->warps = warps0;
        k->auto_seg = auto0;
        k->overlap = overlap0;
        k->resident_blocks = 0;
        return st;
    }
    k->C = C0;
    k->seg_h = best_seg;
    k->warps = best_warps;
    k->overlap = best_overlap;
    k->auto_seg = false;
    k->resident_blocks = 0;
    drop_graph(k);
    TSB_CHECK(k, cudaMemcpyAsync(k->scal, &saved, sizeof saved, cudaMemcpyHostToDevice, k->stream));
    TSB_CHECK(k, cudaStreamSynchronize(k->stream));
    return launch_step(k, 0, true);  // resident grid of the chosen shape
}

int ts_b200_host_alloc(void **ptr, size_t bytes) {
    if (!ptr) return TS_B200_INVALID_ARGUMENT;
    cudaError_t e = cudaHostAlloc(ptr, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR;
    }
    return TS_B200_OK;
}

int ts_b200_host_free(void *ptr) {
    if (!ptr) return TS_B200_OK;
    return cudaFreeHost(ptr) == cudaSuccess ? TS_B200_OK : TS_B200_CUDA_ERROR;
}

}  // extern "C"
