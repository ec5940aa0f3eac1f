// pv_invariants.cu — invariants of the vortex system on the GPU.
//
// Replaces computeMoments / computeInvariants and the three Hamiltonians of the reference
// (src/compute.cpp:11-27, 134-163, 174-202, 262-285), which the reference evaluates serially on
// the host even with its CUDA backend (src/backend_cuda.cu:245-247).
//
//   * moments: one pass over the vortices, per-thread Neumaier-compensated sums;
//   * Hamiltonian: upper-triangular 128 x 128 tiles of the pair matrix (blocks below the diagonal
//     exit at once), per-thread compensated sums, per-block (hi, lo) partials;
//   * a single-block pass adds the block partials in fixed order, so the result is deterministic
//     and independent of scheduling.
#include "pv_internal.h"

namespace pvb {

namespace {
constexpr int kHT = 128;                // Hamiltonian tile edge (threads per block)
constexpr int kMomentBlocks = 256;

// Neumaier's improvement of Kahan summation: s + c carries the sum with the rounding error of
// every addition accumulated in c.
struct CSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        const double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

__constant__ double c_sech[65];   // 1/cosh(2 pi m), m = 0..64
__constant__ double c_tanh2[65];  // tanh(2 pi m)^2

__device__ __forceinline__ double block_sum_fixed(double v, double *sh) {
    // fixed-order tree: warp shuffles then one warp over the warp sums
    for (int off = 16; off > 0; off >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0) {
        r = lane < static_cast<int>(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1)
            r += __shfl_down_sync(0xffffffffu, r, off);
    }
    __syncthreads();
    return r;
}

// scratch layout: [0, 4*kMomentBlocks) moment partials (4 per block),
//                 [4*kMomentBlocks, ...) Hamiltonian partials (2 per tile: hi, lo)
__global__ void __launch_bounds__(256)
    moments_kernel(const double *x, const double *y, const double *g, size_t n, double *part,
                   int *status) {
    __shared__ double sh[32];
    CSum c, ix, iy, l;
    bool bad = false;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const double gi = g[i], xi = x[i], yi = y[i];
        if (!isfinite(gi) || !isfinite(xi) || !isfinite(yi))
            bad = true;
        c.add(gi);
        ix.add(gi * xi);
        iy.add(gi * yi);
        l.add(gi * fma(xi, xi, yi * yi));
    }
    if (bad)
        set_status(status, ST_NONFINITE_POSITION);
    const double m0 = block_sum_fixed(c.value(), sh);
    const double m1 = block_sum_fixed(ix.value(), sh);
    const double m2 = block_sum_fixed(iy.value(), sh);
    const double m3 = block_sum_fixed(l.value(), sh);
    if (threadIdx.x == 0) {
        part[4 * blockIdx.x + 0] = m0;
        part[4 * blockIdx.x + 1] = m1;
        part[4 * blockIdx.x + 2] = m2;
        part[4 * blockIdx.x + 3] = m3;
    }
}

// Pair energies (the sum that the reference multiplies by -1/(4 pi)):
//   infinite: G_i G_j log(r^2 + eps^2)
//   periodic: G_i G_j [ -x^2/(2 pi) + log D_0 + log prod_{m=1..M} D_m D_-m / cosh^2(2 pi m) ]
//             with D_m D_-m / cosh^2 a = (cosh x^ sech a - cos y^)^2 + tanh^2 a sin^2 y^, which is
//             the reference's sum over m of log(den_m) - logCosh(2 pi m) (src/compute.cpp:186-196)
//   disk:     G_i G_j log(|z_i - z_j|^2 R^2 / ((R^2 - z_i.z_j)^2 + (z_i x z_j)^2))
// plus, for the disk, the self terms -G_i^2 log((R^2 - r_i^2)/R) (entered with the sign that makes
// the final -sum/(4 pi) equal the reference).
template <int GEO>
__global__ void __launch_bounds__(kHT)
    hamiltonian_kernel(const double *x, const double *y, const double *g, size_t n,
                       GeometryConsts gc, double *part, int *status) {
    const int I = blockIdx.y, J = blockIdx.x;
    const size_t tile_index = static_cast<size_t>(I) * gridDim.x + J;
    __shared__ double sx[kHT], sy[kHT], sg[kHT];
    __shared__ double sh[32];
    CSum acc;
    if (J >= I) {
        const size_t i = static_cast<size_t>(I) * kHT + threadIdx.x;
        const size_t j0 = static_cast<size_t>(J) * kHT;
        const size_t jl = j0 + threadIdx.x;
        sx[threadIdx.x] = jl < n ? x[jl] : 0.0;
        sy[threadIdx.x] = jl < n ? y[jl] : 0.0;
        sg[threadIdx.x] = jl < n ? g[jl] : 0.0;
        __syncthreads();
        if (i < n) {
            const double xi = x[i], yi = y[i], gi = g[i];
            const int jcount = static_cast<int>(min(static_cast<size_t>(kHT), n - j0));
            const int jstart = (I == J) ? static_cast<int>(threadIdx.x) + 1 : 0;
            if (GEO == GEO_DISK && I == J) {
                const double ri2 = __dadd_rn(__dmul_rn(xi, xi), __dmul_rn(yi, yi));
                if (ri2 >= gc.radius2)
                    set_status(status, ST_OUTSIDE_DISK_H);
                acc.add(-(gi * gi) * log(__ddiv_rn(gc.radius2 - ri2, gc.radius)));
            }
            for (int jj = jstart; jj < jcount; ++jj) {
                const double xj = sx[jj], yj = sy[jj], gj = sg[jj];
                double term;
                if (GEO == GEO_INFINITE) {
                    const double dx = xi - xj, dy = yi - yj;
                    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), gc.eps2);
                    if (r2 == 0.0)
                        set_status(status, ST_COINCIDENT);
                    term = log(r2);
                } else if (GEO == GEO_PERIODIC) {
                    const double xh = gc.wave * exact_remainder(xi - xj, gc.lx, gc.inv_lx, gc.half_lx);
                    const double yh = gc.wave * exact_remainder(yi - yj, gc.ly, gc.inv_ly, gc.half_ly);
                    double shx, chx, snx, csx, shy, chy, sny, csy;
                    sinh_cosh_sin_cos(0.5 * xh, shx, chx, snx, csx);
                    sinh_cosh_sin_cos(0.5 * yh, shy, chy, sny, csy);
                    const double d0 = 2.0 * fma(shx, shx, sny * sny);
                    if (d0 == 0.0)
                        set_status(status, ST_COINCIDENT);
                    const double cosh_x = fma(2.0 * shx, shx, 1.0);
                    const double cos_y = fma(-2.0 * sny, sny, 1.0);
                    const double sin_y = 2.0 * sny * csy;
                    const double s2 = sin_y * sin_y;
                    double prod = 1.0;
                    for (int m = 1; m <= gc.image_layers; ++m) {
                        const double q = fma(cosh_x, c_sech[m], -cos_y);
                        prod *= fma(q, q, c_tanh2[m] * s2);
                    }
                    term = -xh * xh / (2.0 * kPi) + log(d0) + log(prod);
                } else {
                    const double dx = xi - xj, dy = yi - yj;
                    const double num = (dx * dx + dy * dy) * gc.radius2;
                    const double dot = xi * xj + yi * yj;
                    const double cross = yi * xj - xi * yj;
                    const double den = (gc.radius2 - dot) * (gc.radius2 - dot) + cross * cross;
                    if (num == 0.0)
                        set_status(status, ST_COINCIDENT);
                    term = log(num / den);
                }
                acc.add((gi * gj) * term);
            }
        }
    }
    const double hi = block_sum_fixed(acc.s, sh);
    const double lo = block_sum_fixed(acc.c, sh);
    if (threadIdx.x == 0) {
        part[2 * tile_index] = hi;
        part[2 * tile_index + 1] = lo;
    }
}

// One block: fixed-order compensated sum of the moment partials and Hamiltonian partials.
__global__ void __launch_bounds__(1024)
    finalize_kernel(const double *part, int moment_blocks, size_t tiles, double *out, int *status,
                    int *status_h) {
    __shared__ double sh[32];
    for (int k = 0; k < 4; ++k) {
        CSum c;
        for (int b = threadIdx.x; b < moment_blocks; b += blockDim.x)
            c.add(part[4 * b + k]);
        const double hi = block_sum_fixed(c.s, sh);
        const double lo = block_sum_fixed(c.c, sh);
        if (threadIdx.x == 0) {
            out[k] = hi + lo;
            if (!isfinite(out[k]))
                set_status_if_clean(status, ST_NONFINITE_MOMENT);
        }
    }
    const double *hp = part + 4 * moment_blocks;
    CSum h;
    for (size_t t = threadIdx.x; t < tiles; t += blockDim.x) {
        h.add(hp[2 * t]);
        h.add(hp[2 * t + 1]);
    }
    const double hi = block_sum_fixed(h.s, sh);
    const double lo = block_sum_fixed(h.c, sh);
    if (threadIdx.x == 0) {
        const double hamiltonian = -(hi + lo) / (4.0 * kPi);
        out[4] = hamiltonian;
        if (!isfinite(hamiltonian))
            set_status_if_clean(status_h, ST_NONFINITE_HAMILTONIAN);
    }
}

bool g_tables_ready[64] = {};
} // namespace

size_t invariants_scratch_doubles(size_t n, int) {
    const size_t nt = (n + kHT - 1) / kHT;
    return 4 * static_cast<size_t>(kMomentBlocks) + 2 * (nt > 0 ? nt * nt : 1);
}

cudaError_t launch_invariants(const double *x, const double *y, const double *gamma, size_t n,
                              const GeometryConsts &g, double *scratch, double *out, int *status,
                              int *status_h, cudaStream_t stream) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (g.geometry == GEO_PERIODIC && dev >= 0 && dev < 64 && !g_tables_ready[dev]) {
        double sech[65], tanh2[65];
        for (int m = 0; m <= 64; ++m) {
            const double a = 2.0 * kPi * m;
            sech[m] = 1.0 / cosh(a);
            const double t = tanh(a);
            tanh2[m] = t * t;
        }
        cudaError_t e = cudaMemcpyToSymbol(c_sech, sech, sizeof(sech));
        if (e == cudaSuccess)
            e = cudaMemcpyToSymbol(c_tanh2, tanh2, sizeof(tanh2));
        if (e != cudaSuccess)
            return e;
        g_tables_ready[dev] = true;
    }
    moments_kernel<<<kMomentBlocks, 256, 0, stream>>>(x, y, gamma, n, scratch, status);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    const size_t nt = (n + kHT - 1) / kHT;
    size_t tiles = 0;
    if (nt > 0) {
        const dim3 grid(static_cast<unsigned>(nt), static_cast<unsigned>(nt));
        double *hp = scratch + 4 * kMomentBlocks;
        switch (g.geometry) {
        case GEO_INFINITE:
            hamiltonian_kernel<GEO_INFINITE><<<grid, kHT, 0, stream>>>(x, y, gamma, n, g, hp, status_h);
            break;
        case GEO_PERIODIC:
            hamiltonian_kernel<GEO_PERIODIC><<<grid, kHT, 0, stream>>>(x, y, gamma, n, g, hp, status_h);
            break;
        default:
            hamiltonian_kernel<GEO_DISK><<<grid, kHT, 0, stream>>>(x, y, gamma, n, g, hp, status_h);
            break;
        }
        if ((e = cudaGetLastError()) != cudaSuccess)
            return e;
        tiles = nt * nt;
    }
    finalize_kernel<<<1, 1024, 0, stream>>>(scratch, kMomentBlocks, tiles, out, status, status_h);
    return cudaGetLastError();
}

} // namespace pvb
