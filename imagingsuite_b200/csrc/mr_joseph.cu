// Differentiable parallel-beam projector pair (sm_100a).
//
// Forward: the Joseph ray-driven projector of LinearForwardProjector::project
// (ReconAlgorithms/linearforwardprojector.cpp:15-144), applied to every slice z of a volume
// [nz][n][n] (x fastest) with a per-slice detector centre c_z = centre + tan_tilt (z - pivot)
// (the reference fixes the centre at R/2: centre = nu/2, tan_tilt = 0 reproduces it). For an
// angle with |sin| > sqrt(1/2) a ray steps along x (major index k) and interpolates linearly
// along y at f = beta + k alpha; otherwise it steps along y and interpolates along x. A
// sample counts when 0 <= f < n - 1; the ray sum is scaled by 1/|sin| (or 1/|cos|).
//
// Adjoint: the exact transpose, voxel-driven. A voxel (x, y) receives weight (1 - w) from the
// rays whose sample at its major index falls in [minor, minor + 1) and w from those in
// [minor - 1, minor). Those rays form the interval rc -+ |s| of detector positions (s = 1/inv);
// the candidates are the integers within it widened by a margin of 0.02 + 1e-5 (n + nu) bins,
// far above the float error of the bracket and of a sample position (which grows with the
// magnitudes involved: below 4e-4 bin for n, nu up to 4096), and every candidate's sample position is recomputed with the forward's own
// expression (joseph_pos), so forward and adjoint use bit-identical weights and the same
// sample set: <A x, y> = <x, A^T y> up to the summation order.
//
// Centre derivative: d(A x)/d centre = -inv d sum_k (s1 - s0) for a ray (the interpolation
// is linear within a pixel), produced by the forward kernel on request; per-slice dot
// products with a residual give the gradients of 1/2 |A x - p|^2 with respect to the centre
// and, through c_z, the tilt.
//
// Per-angle geometry (alpha, 1/sin or 1/cos, weight, ray offset) is computed in FP64 on the
// host and rounded once to float.
#include "mr_common.cuh"

#include <cmath>
#include <cstring>

namespace mr {
namespace joseph {

struct Angle {
    float major_y; // 1: rays step along y
    float alpha, inv, d, rho_off;
    float s;       // 1 / inv (sin or cos), for the adjoint's ray bracket
    float pad[2];
};

static_assert(sizeof(Angle) == 32, "Angle layout");

// Sample position of ray r at major index k (shared by forward, adjoint and derivative).
__device__ __forceinline__ float joseph_beta(int r, float cz, const Angle &g)
{
    return __fmul_rn(__fsub_rn(__fsub_rn(static_cast<float>(r), cz), g.rho_off), g.inv);
}

__device__ __forceinline__ float joseph_pos(float beta, int k, const Angle &g)
{
    return __fmaf_rn(static_cast<float>(k), g.alpha, beta);
}

// Range of major indices whose sample may lie in [0, n - 1), widened by one on each side
// (the exact test is applied per sample).
__device__ __forceinline__ void major_range(float beta, float alpha, int n, int &k0, int &k1)
{
    k0 = 0;
    k1 = n;
    if (fabsf(alpha) > 1e-6f) {
        const float a = (0.0f - beta) / alpha, b = (static_cast<float>(n - 1) - beta) / alpha;
        const float lo = fminf(a, b), hi = fmaxf(a, b);
        k0 = max(0, static_cast<int>(floorf(fmaxf(lo, -1.0f))) - 1);
        k1 = min(n, static_cast<int>(ceilf(fminf(hi, static_cast<float>(n) + 1.0f))) + 2);
    }
}

// One thread per ray (r, z, t). vol: [nz][n][n] slices; volt: the same slices transposed
// ([nz][x][y]), so that both stepping directions read consecutive minor positions. The grid
// runs the angles of a slice together (t = blockIdx.y, z = blockIdx.z), so the resident
// blocks read a few slices from L2 instead of streaming the volume from DRAM per angle.
__global__ void __launch_bounds__(128) k_forward(const float *__restrict__ vol, const float *__restrict__ volt, int n,
                                                 int nz, const Angle *__restrict__ ang, int nu, float centre,
                                                 float tan_tilt, float pivot, float *__restrict__ proj,
                                                 float *__restrict__ dproj)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x, t = blockIdx.y, z = blockIdx.z;
    if (r >= nu) return;
    const Angle g = ang[t];
    const float cz = __fmaf_rn(tan_tilt, static_cast<float>(z) - pivot, centre);
    const float beta = joseph_beta(r, cz, g);
    // plane[k][minor]: y-stepping rays read vol rows, x-stepping rays read volt rows
    const float *plane = (g.major_y != 0.0f ? vol : volt) + static_cast<size_t>(z) * n * n;
    int k0, k1;
    major_range(beta, g.alpha, n, k0, k1);
    float sum = 0.0f, dsum = 0.0f;
    const float lim = static_cast<float>(n - 1);
    for (int k = k0; k < k1; ++k) {
        const float f = joseph_pos(beta, k, g);
        if (!(f >= 0.0f && f < lim)) continue;
        const int i0 = static_cast<int>(f);
        const float w = f - static_cast<float>(i0);
        const float *row = plane + static_cast<size_t>(k) * n + i0;
        const float s0 = __ldg(row), s1 = __ldg(row + 1);
        sum = __fmaf_rn(w, s1 - s0, sum + s0);
        dsum += s1 - s0;
    }
    const size_t o = (static_cast<size_t>(t) * nz + z) * nu + r;
    proj[o] = sum * g.d;
    if (dproj) dproj[o] = -dsum * g.inv * g.d;
}

// One thread per voxel (x, y, z): gather over angles and candidate rays. The per-angle
// parameters are staged in shared memory in chunks of kAngleChunk.
constexpr int kAngleChunk = 256;

__global__ void __launch_bounds__(128) k_adjoint(const float *__restrict__ proj, int n, int nz,
                                                 const Angle *__restrict__ ang, int nproj, int nu, float centre,
                                                 float tan_tilt, float pivot, float margin, int accumulate,
                                                 float *__restrict__ vol)
{
    __shared__ Angle sa[kAngleChunk];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
    const float cz = __fmaf_rn(tan_tilt, static_cast<float>(z) - pivot, centre);
    const float lim = static_cast<float>(n - 1);
    float acc = 0.0f;
    for (int t0 = 0; t0 < nproj; t0 += kAngleChunk) {
        const int nt = min(kAngleChunk, nproj - t0);
        __syncthreads();
        for (int i = threadIdx.x; i < nt; i += blockDim.x) sa[i] = ang[t0 + i];
        __syncthreads();
        if (x >= n) continue;
        for (int tt = 0; tt < nt; ++tt) {
            const Angle g = sa[tt];
            const bool my = g.major_y != 0.0f;
            const int k = my ? y : x, minor = my ? x : y;
            // f(r) = (r - cz - rho_off) inv + k alpha; rays with f in [minor - 1, minor + 1)
            const float rc = (static_cast<float>(minor) - static_cast<float>(k) * g.alpha) * g.s + cz + g.rho_off;
            const float hw = fabsf(g.s) + margin;
            // the integers within [rc - hw, rc + hw]: 2|s| + 1 <= 3 rays, a fourth only when the
            // margin exceeds half a bin (very large sizes)
            const int r0 = max(0, static_cast<int>(ceilf(rc - hw))), r1 = min(nu - 1, static_cast<int>(floorf(rc + hw)));
            const float *p = proj + (static_cast<size_t>(t0 + tt) * nz + z) * nu;
            auto ray = [&](int r) {
                const float f = joseph_pos(joseph_beta(r, cz, g), k, g);
                if (!(f >= 0.0f && f < lim)) return;
                const int i0 = static_cast<int>(f);
                const float w = f - static_cast<float>(i0);
                if (i0 == minor) acc = __fmaf_rn((1.0f - w) * g.d, __ldg(p + r), acc);
                else if (i0 == minor - 1) acc = __fmaf_rn(w * g.d, __ldg(p + r), acc);
            };
#pragma unroll
            for (int j = 0; j < 3; ++j)
                if (r0 + j <= r1) ray(r0 + j);
            for (int r = r0 + 3; r <= r1; ++r) ray(r);
        }
    }
    if (x >= n) return;
    float *o = vol + (static_cast<size_t>(z) * n + y) * n + x;
    *o = accumulate ? *o + acc : acc;
}

// [nz][n][n] -> [nz][x][y]
__global__ void k_transpose(const float *__restrict__ in, int n, float *__restrict__ out)
{
    __shared__ float tile[32][33];
    const int z = blockIdx.z;
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    const float *src = in + static_cast<size_t>(z) * n * n;
    float *dst = out + static_cast<size_t>(z) * n * n;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int y = by + j, x = bx + threadIdx.x;
        if (x < n && y < n) tile[j][threadIdx.x] = src[static_cast<size_t>(y) * n + x];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int x = bx + j, y = by + threadIdx.x;
        if (x < n && y < n) dst[static_cast<size_t>(x) * n + y] = tile[threadIdx.x][j];
    }
}

// out[z] = sum over (t, r) of a[t][z][r] * b[t][z][r], FP64 accumulation.
__global__ void k_slice_dot(const float *__restrict__ a, const float *__restrict__ b, int nproj, int nz, int nu,
                            double *__restrict__ out)
{
    const int z = blockIdx.x;
    double s = 0.0;
    for (int i = threadIdx.x; i < nproj * nu; i += blockDim.x) {
        const int t = i / nu, r = i % nu;
        const size_t o = (static_cast<size_t>(t) * nz + z) * nu + r;
        s += static_cast<double>(a[o]) * b[o];
    }
    __shared__ double red[32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) out[z] = s;
    }
}

} // namespace joseph
} // namespace mr

using namespace mr;
using namespace mr::joseph;

extern "C" {

mr_status mr_joseph_geometry(const float *angles_h, size_t nproj, size_t n, float *params_h)
{
    MR_TRACE();
    if (nproj && (!angles_h || !params_h)) return fail(MR_ERR_ARGUMENT, "mr_joseph_geometry: null pointer");
    if (n < 2) return fail(MR_ERR_ARGUMENT, "mr_joseph_geometry: slice size below 2");
    const double kPi = 3.1415926535897932384626433832795028841971693993751;
    const double x_min = -static_cast<double>(static_cast<long>(n / 2));
    for (size_t t = 0; t < nproj; ++t) {
        const double th = static_cast<double>(angles_h[t]) * kPi / 180.0;
        const double sn = std::sin(th), cs = std::cos(th);
        Angle g{};
        g.rho_off = static_cast<float>(x_min * (cs + sn));
        if (std::fabs(sn) > std::sqrt(0.5)) {
            g.major_y = 0.0f;
            g.alpha = static_cast<float>(-cs / sn);
            g.inv = static_cast<float>(1.0 / sn);
            g.s = static_cast<float>(sn);
            g.d = static_cast<float>(1.0 / std::fabs(sn));
        } else {
            g.major_y = 1.0f;
            g.alpha = static_cast<float>(-sn / cs);
            g.inv = static_cast<float>(1.0 / cs);
            g.s = static_cast<float>(cs);
            g.d = static_cast<float>(1.0 / std::fabs(cs));
        }
        std::memcpy(params_h + t * 8, &g, sizeof(Angle));
    }
    return MR_OK;
}

mr_status mr_joseph_forward(const float *vol_d, float *volt_d, size_t n, size_t nz, const float *params_d,
                            size_t nproj, size_t nu, float centre, float tan_tilt, float pivot, float *proj_d,
                            float *dproj_d, void *stream)
{
    MR_TRACE();
    if (!vol_d || !volt_d || !params_d || !proj_d) return fail(MR_ERR_ARGUMENT, "mr_joseph_forward: null pointer");
    if (n < 2 || n > 65536 || nz == 0 || nz > 65535 || nu == 0 || nproj == 0 || nproj > 65535)
        return fail(MR_ERR_ARGUMENT, "mr_joseph_forward: unsupported size");
    cudaStream_t s = as_stream(stream);
    dim3 tb(32, 8), tg(div_up(n, 32), div_up(n, 32), static_cast<unsigned>(nz));
    k_transpose<<<tg, tb, 0, s>>>(vol_d, static_cast<int>(n), volt_d);
    mr_status st = check_launch("k_transpose");
    if (st != MR_OK) return st;
    dim3 grid(div_up(nu, 128), static_cast<unsigned>(nproj), static_cast<unsigned>(nz));
    k_forward<<<grid, 128, 0, s>>>(vol_d, volt_d, static_cast<int>(n), static_cast<int>(nz),
                                   reinterpret_cast<const Angle *>(params_d), static_cast<int>(nu), centre, tan_tilt,
                                   pivot, proj_d, dproj_d);
    return check_launch("k_forward");
}

mr_status mr_joseph_adjoint(const float *proj_d, size_t n, size_t nz, const float *params_d, size_t nproj, size_t nu,
                            float centre, float tan_tilt, float pivot, int accumulate, float *vol_d, void *stream)
{
    MR_TRACE();
    if (!proj_d || !params_d || !vol_d) return fail(MR_ERR_ARGUMENT, "mr_joseph_adjoint: null pointer");
    if (n < 2 || n > 65535 || nz == 0 || nz > 65535 || nu == 0 || nproj == 0 || nproj > 65535)
        return fail(MR_ERR_ARGUMENT, "mr_joseph_adjoint: unsupported size");
    dim3 grid(div_up(n, 128), static_cast<unsigned>(n), static_cast<unsigned>(nz));
    k_adjoint<<<grid, 128, 0, as_stream(stream)>>>(proj_d, static_cast<int>(n), static_cast<int>(nz),
                                                   reinterpret_cast<const Angle *>(params_d),
                                                   static_cast<int>(nproj), static_cast<int>(nu), centre, tan_tilt,
                                                   pivot, 0.02f + 1e-5f * static_cast<float>(n + nu), accumulate,
                                                   vol_d);
    return check_launch("k_adjoint");
}

mr_status mr_slice_dot(const float *a_d, const float *b_d, size_t nproj, size_t nz, size_t nu, double *out_d,
                       void *stream)
{
    MR_TRACE();
    if (!a_d || !b_d || !out_d) return fail(MR_ERR_ARGUMENT, "mr_slice_dot: null pointer");
    if (nz == 0 || nz > 65535 || nproj * nu > 0x7fffffff) return fail(MR_ERR_ARGUMENT, "mr_slice_dot: unsupported size");
    k_slice_dot<<<static_cast<unsigned>(nz), 512, 0, as_stream(stream)>>>(a_d, b_d, static_cast<int>(nproj),
                                                                          static_cast<int>(nz), static_cast<int>(nu),
                                                                          out_d);
    return check_launch("k_slice_dot");
}

} // extern "C"
