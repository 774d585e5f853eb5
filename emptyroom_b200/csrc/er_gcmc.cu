// er_gcmc.cu -- GCMC guest-framework energies looked up in a device-resident
// grid (er_grid_interp).
//
// The reference's GCMC code (src/gcmc.cc) never evaluates the pair sum for a
// guest: it interpolates the energy grid trilinearly (GuestFrameworkEnergy,
// src/gcmc.cc:145-177) at the guest's wrapped fractional position
// (WrapToInterval(x, 1), src/gcmc.cc:74-77, at the call sites :191-194,
// :470-473, :530-533, :588-591), with spacing 1 / (N - 1) (:343-345). Here
// one thread evaluates one point with the same FP64 expressions in the same
// order (no contraction), so a point's result is bit for bit the reference
// function's on the same grid values; grids may be FP32 (as er_grid writes
// them, widened exactly) or FP64. Pocket points blocked to 1e13 interpolate
// as in the reference.
#include <math.h>

#include "er_ctx.h"

namespace er {

__device__ __forceinline__ double wrap1(double x) {
    // WrapToInterval(x, 1.0) = x - 1.0 * floor(x / 1.0)
    return __dsub_rn(x, __dmul_rn(1.0, floor(__ddiv_rn(x, 1.0))));
}

template <typename G>
__global__ void __launch_bounds__(256) grid_interp_kernel(const G* __restrict__ grid, int nx,
                                                          int ny, int nz,
                                                          const double* __restrict__ pts,
                                                          int64_t n, double* __restrict__ out) {
    const double dx = __ddiv_rn(1.0, (double)(nx - 1));
    const double dy = __ddiv_rn(1.0, (double)(ny - 1));
    const double dz = __ddiv_rn(1.0, (double)(nz - 1));
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const double x = wrap1(pts[3 * q]), y = wrap1(pts[3 * q + 1]), z = wrap1(pts[3 * q + 2]);
        // lower corner, clamped to N - 2 (the reference would read past the
        // grid where x / dx rounds up to N - 1 for x just below 1)
        const int i = min((int)floor(__ddiv_rn(x, dx)), nx - 2);
        const int j = min((int)floor(__ddiv_rn(y, dy)), ny - 2);
        const int k = min((int)floor(__ddiv_rn(z, dz)), nz - 2);
        const double xd = __ddiv_rn(__dsub_rn(x, __dmul_rn((double)i, dx)), dx);
        const double yd = __ddiv_rn(__dsub_rn(y, __dmul_rn((double)j, dy)), dy);
        const double zd = __ddiv_rn(__dsub_rn(z, __dmul_rn((double)k, dz)), dz);
        auto g = [&](int a, int b, int c) {
            return (double)grid[(size_t)c + (size_t)b * nz + (size_t)a * ny * nz];
        };
        const double ox = __dsub_rn(1.0, xd);
        const double c00 = __dadd_rn(__dmul_rn(g(i, j, k), ox), __dmul_rn(xd, g(i + 1, j, k)));
        const double c10 =
            __dadd_rn(__dmul_rn(g(i, j + 1, k), ox), __dmul_rn(xd, g(i + 1, j + 1, k)));
        const double c01 =
            __dadd_rn(__dmul_rn(g(i, j, k + 1), ox), __dmul_rn(xd, g(i + 1, j, k + 1)));
        const double c11 =
            __dadd_rn(__dmul_rn(g(i, j + 1, k + 1), ox), __dmul_rn(xd, g(i + 1, j + 1, k + 1)));
        const double oy = __dsub_rn(1.0, yd);
        const double c0 = __dadd_rn(__dmul_rn(c00, oy), __dmul_rn(c10, yd));
        const double c1 = __dadd_rn(__dmul_rn(c01, oy), __dmul_rn(c11, yd));
        out[q] = __dadd_rn(__dmul_rn(c0, __dsub_rn(1.0, zd)), __dmul_rn(c1, zd));
    }
}

static bool is_device_ptr(const void* p) {
    cudaPointerAttributes attr;
    const bool dev = cudaPointerGetAttributes(&attr, p) == cudaSuccess &&
                     (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    return dev;
}

}  // namespace er

using namespace er;

extern "C" int er_grid_interp(er_ctx* ctx, const void* grid, int nx, int ny, int nz, int flags,
                              const double* pts, int64_t n, double* out) {
    if (!ctx || !grid || (n > 0 && (!pts || !out)) || n < 0) return ER_ERR_INVALID;
    if (nx < 2 || ny < 2 || nz < 2)
        return set_error(ctx, ER_ERR_INVALID, "grid_interp: nx, ny, nz must be >= 2");
    if ((flags & ~ER_INTERP_GRID_F64) != 0)
        return set_error(ctx, ER_ERR_INVALID, "grid_interp: unknown flags");
    if (n == 0) return ER_OK;
    ER_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!is_device_ptr(grid))
        return set_error(ctx, ER_ERR_INVALID, "grid_interp: grid must be device memory");
    cudaStream_t st = ctx->stream;
    const bool pts_dev = is_device_ptr(pts), out_dev = is_device_ptr(out);
    const double* d_pts = pts;
    double* d_out = out;
    const size_t b_pts = (size_t)n * 3 * sizeof(double), b_out = (size_t)n * sizeof(double);
    if (!pts_dev || !out_dev) {
        if (ctx->interp.ensure((pts_dev ? 0 : b_pts) + (out_dev ? 0 : b_out)) != ER_OK)
            return set_error(ctx, ER_ERR_NOMEM, "grid_interp: staging allocation failed");
        char* b = (char*)ctx->interp.ptr;
        if (!pts_dev) {
            d_pts = (const double*)b;
            ER_CUDA(ctx, cudaMemcpyAsync(b, pts, b_pts, cudaMemcpyHostToDevice, st));
            b += b_pts;
        }
        if (!out_dev) d_out = (double*)b;
    }
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8);
    if (flags & ER_INTERP_GRID_F64)
        grid_interp_kernel<double><<<blocks, 256, 0, st>>>((const double*)grid, nx, ny, nz, d_pts,
                                                           n, d_out);
    else
        grid_interp_kernel<float><<<blocks, 256, 0, st>>>((const float*)grid, nx, ny, nz, d_pts,
                                                          n, d_out);
    ER_CUDA(ctx, cudaGetLastError());
    if (!out_dev) ER_CUDA(ctx, cudaMemcpyAsync(out, d_out, b_out, cudaMemcpyDeviceToHost, st));
    ER_CUDA(ctx, cudaStreamSynchronize(st));
    return ER_OK;
}
