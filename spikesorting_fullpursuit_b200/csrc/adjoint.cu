// adjoint.cu -- residual energy of a fixed spike assignment and its gradient.
//
// Template refinement at fixed assignments (no counterpart in the reference):
//     r(c, x) = v(c, x) - sum_k a_k * T~_k(c, x - s_k)
//     E       = sum_{c,x} r(c, x)^2
// where spike k has onset s_k (the pursuit's event index), label l_k, amplitude
// a_k and fractional shift tau_k in (-1, 1) samples, and T~ is template l_k moved
// right by tau_k with linear interpolation:
//     u = |tau|, dir = tau >= 0 ? -1 : +1
//     T~(c, j) = (1 - u) T(c, j) + u T(c, j + dir),   j in [-1, W]   (T = 0 outside [0, W))
// Samples outside [0, N) are not modelled.  Gradients:
//     dE/da_k     = -2 sum_{c,j} T~_k(c, j) r(c, s_k + j)
//     dE/dtau_k   = -2 a_k sgn(tau_k) sum_{c,j} (T(c, j + dir) - T(c, j)) r(c, s_k + j)
//                   (sgn(0) = +1: the tau >= 0 branch)
//     dE/dT_l(c,i)= -2 sum_{k: l_k = l} a_k ((1 - u) r(c, s_k + i) + u r(c, s_k + i - dir))
// Nothing is stored between the loss and the gradient: each CTA rebuilds its
// spike's residual tile r(:, [s_k - 1, s_k + W]) in FP64 from the voltage and
// every spike whose support meets the tile (spikes sorted by onset; the
// neighbours are found by binary search).  Sums run in FP64; template gradients
// accumulate with FP64 atomics.  The loss is sum v^2 plus, for every modelled
// sample, r^2 - v^2 counted once, by the first spike (in onset order) whose
// support holds it.
#include <cub/cub.cuh>

#include "fbp_internal.cuh"

namespace fbp {
namespace {

constexpr int kAdjThreads = 128;

struct AdjArgs {
    uint32_t C, N, M, W;
    const float* V;        // [C][N]
    const float* T;        // [M][C][W]
    const uint32_t* idx;   // [n] onsets, ascending
    const uint32_t* lab;   // [n]
    const float* amp;      // [n]
    const float* tau;      // [n]
    uint32_t n;
};

__device__ __forceinline__ double tshift(const float* Tc, int W, double u, int dir, int j)
{
    const double a = (j >= 0 && j < W) ? (double)Tc[j] : 0.0;
    const int jj = j + dir;
    const double b = (jj >= 0 && jj < W) ? (double)Tc[jj] : 0.0;
    return (1.0 - u) * a + u * b;
}

// first spike with onset >= key
__device__ uint32_t lower_bound(const uint32_t* idx, uint32_t n, int64_t key)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((int64_t)idx[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Residual tile of spike k: r[c][x - (s_k - 1)] for x in [s_k - 1, s_k + W], all
// channels, in FP64 shared memory (samples outside [0, N) left at 0).
__device__ void residual_tile(const AdjArgs& A, uint32_t k, double* r)
{
    const int W = (int)A.W, TL = W + 2;
    const int64_t x0 = (int64_t)A.idx[k] - 1;
    for (int e = threadIdx.x; e < (int)A.C * TL; e += blockDim.x) {
        const int c = e / TL, q = e - c * TL;
        const int64_t x = x0 + q;
        r[e] = (x >= 0 && x < (int64_t)A.N) ? (double)A.V[(uint64_t)c * A.N + x] : 0.0;
    }
    __syncthreads();
    const uint32_t k_lo = lower_bound(A.idx, A.n, (int64_t)A.idx[k] - W - 1);
    const uint32_t k_hi = lower_bound(A.idx, A.n, (int64_t)A.idx[k] + W + 2);
    for (uint32_t kk = k_lo; kk < k_hi; ++kk) {
        const uint32_t l = A.lab[kk];
        if (l >= A.M) continue;
        const double a = A.amp[kk], t = A.tau[kk];
        const double u = t >= 0.0 ? t : -t;
        const int dir = t >= 0.0 ? -1 : 1;
        const int64_t off = (int64_t)A.idx[kk] - x0;   // tile column of the neighbour's j = 0
        for (int e = threadIdx.x; e < (int)A.C * TL; e += blockDim.x) {
            const int c = e / TL, q = e - c * TL;
            const int64_t x = x0 + q;
            const int j = (int)(q - off);
            if (j < -1 || j > W || x < 0 || x >= (int64_t)A.N) continue;
            r[e] -= a * tshift(A.T + ((uint64_t)l * A.C + c) * A.W, W, u, dir, j);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kAdjThreads) adjoint_loss_kernel(AdjArgs A, double* loss)
{
    extern __shared__ double r[];
    typedef cub::BlockReduce<double, kAdjThreads> R;
    __shared__ typename R::TempStorage tmp;
    const int W = (int)A.W, TL = W + 2;
    double acc = 0.0;
    for (uint32_t k = blockIdx.x; k < A.n; k += gridDim.x) {
        __syncthreads();
        residual_tile(A, k, r);
        const int64_t x0 = (int64_t)A.idx[k] - 1;
        // samples owned by this spike: not covered by an earlier one (the previous
        // spike in onset order has the furthest-reaching earlier support)
        const int64_t first = k > 0 ? (int64_t)A.idx[k - 1] + W + 1 : INT64_MIN;
        for (int e = threadIdx.x; e < (int)A.C * TL; e += blockDim.x) {
            const int c = e / TL, q = e - c * TL;
            const int64_t x = x0 + q;
            if (x < 0 || x >= (int64_t)A.N || x < first) continue;
            const double v = A.V[(uint64_t)c * A.N + x];
            acc += r[e] * r[e] - v * v;
        }
    }
    const double s = R(tmp).Sum(acc);
    if (threadIdx.x == 0 && s != 0.0) atomicAdd(loss, s);
}

__global__ void sumsq_kernel(const float* __restrict__ V, uint64_t n, double* out)
{
    typedef cub::BlockReduce<double, 256> R;
    __shared__ typename R::TempStorage tmp;
    double acc = 0.0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const double v = V[i];
        acc += v * v;
    }
    const double s = R(tmp).Sum(acc);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

__global__ void __launch_bounds__(kAdjThreads) adjoint_grad_kernel(AdjArgs A, double scale, double* gT, float* g_amp,
                                                                  float* g_tau)
{
    extern __shared__ double r[];
    typedef cub::BlockReduce<double, kAdjThreads> R;
    __shared__ typename R::TempStorage tmp;
    const int W = (int)A.W, TL = W + 2;
    for (uint32_t k = blockIdx.x; k < A.n; k += gridDim.x) {
        __syncthreads();
        residual_tile(A, k, r);
        const uint32_t l = A.lab[k];
        double da = 0.0, dt = 0.0;
        if (l < A.M) {
            const double a = A.amp[k], t = A.tau[k];
            const double u = t >= 0.0 ? t : -t;
            const int dir = t >= 0.0 ? -1 : 1;
            const double sg = t >= 0.0 ? 1.0 : -1.0;
            for (int e = threadIdx.x; e < (int)A.C * TL; e += blockDim.x) {
                const int c = e / TL, q = e - c * TL;
                const int j = q - 1;
                const float* Tc = A.T + ((uint64_t)l * A.C + c) * A.W;
                const double ts = tshift(Tc, W, u, dir, j);
                const double tj = (j >= 0 && j < W) ? (double)Tc[j] : 0.0;
                const int jj = j + dir;
                const double td = (jj >= 0 && jj < W) ? (double)Tc[jj] : 0.0;
                da += ts * r[e];
                dt += (td - tj) * r[e];
                // template sample i = j: (1 - u) r(s + i) + u r(s + i - dir)
                if (j >= 0 && j < W) {
                    const int q2 = q - dir;   // tile column of s + i - dir, in [0, TL)
                    const double g = (1.0 - u) * r[e] + u * r[c * TL + q2];
                    atomicAdd(&gT[((uint64_t)l * A.C + c) * A.W + j], -2.0 * scale * a * g);
                }
            }
            dt *= sg * a;
        }
        const double sa = R(tmp).Sum(da);
        __syncthreads();
        const double st = R(tmp).Sum(dt);
        if (threadIdx.x == 0) {
            g_amp[k] = (float)(-2.0 * scale * sa);
            g_tau[k] = (float)(-2.0 * scale * st);
        }
    }
}

__global__ void f64_to_f32_kernel(const double* __restrict__ a, float* b, uint64_t n)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

int adj_check(const fbp_dims* d, const float* V, const float* T, const uint32_t* idx, const uint32_t* lab,
              const float* amp, const float* tau, uint32_t n)
{
    if (!d) return fail(FBP_E_ARG, "null dims");
    if (d->n_chans == 0 || d->n_samples == 0 || d->n_templates == 0 || d->template_len == 0)
        return fail(FBP_E_ARG, "invalid dims");
    if ((size_t)d->n_chans * (d->template_len + 2) * sizeof(double) > 200 * 1024)
        return fail(FBP_E_ARG, "channels x template length too large for one residual tile");
    if (!V || !T) return fail(FBP_E_ARG, "null pointer argument");
    if (n > 0 && (!idx || !lab || !amp || !tau)) return fail(FBP_E_ARG, "null spike argument");
    return FBP_OK;
}

AdjArgs adj_args(const fbp_dims* d, const float* V, const float* T, const uint32_t* idx, const uint32_t* lab,
                 const float* amp, const float* tau, uint32_t n)
{
    AdjArgs A;
    A.C = d->n_chans;
    A.N = d->n_samples;
    A.M = d->n_templates;
    A.W = d->template_len;
    A.V = V;
    A.T = T;
    A.idx = idx;
    A.lab = lab;
    A.amp = amp;
    A.tau = tau;
    A.n = n;
    return A;
}

}  // namespace
}  // namespace fbp

using namespace fbp;

extern "C" int fbp_adjoint_loss(const fbp_dims* dims, const float* voltage, const float* templates,
                                const uint32_t* spike_idx, const uint32_t* spike_lab, const float* amplitude,
                                const float* shift, uint32_t n_spikes, double* loss, void* stream)
{
    set_error("");
    const int rc = adj_check(dims, voltage, templates, spike_idx, spike_lab, amplitude, shift, n_spikes);
    if (rc != FBP_OK) return rc;
    if (!loss) return fail(FBP_E_ARG, "null loss");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const AdjArgs A = adj_args(dims, voltage, templates, spike_idx, spike_lab, amplitude, shift, n_spikes);
    FBP_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), st));
    count_launch();
    sumsq_kernel<<<148 * 4, 256, 0, st>>>(voltage, (uint64_t)A.C * A.N, loss);
    if (n_spikes) {
        const size_t smem = (size_t)A.C * (A.W + 2) * sizeof(double);
        FBP_CUDA(allow_max_dyn_smem(adjoint_loss_kernel));
        count_launch();
        adjoint_loss_kernel<<<n_spikes < 148u * 16 ? n_spikes : 148u * 16, kAdjThreads, smem, st>>>(A, loss);
    }
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}

extern "C" int fbp_adjoint_grad(const fbp_dims* dims, const float* voltage, const float* templates,
                                const uint32_t* spike_idx, const uint32_t* spike_lab, const float* amplitude,
                                const float* shift, uint32_t n_spikes, double scale, double* grad_templates64,
                                float* grad_templates, float* grad_amplitude, float* grad_shift, void* stream)
{
    set_error("");
    const int rc = adj_check(dims, voltage, templates, spike_idx, spike_lab, amplitude, shift, n_spikes);
    if (rc != FBP_OK) return rc;
    if (!grad_templates64 || !grad_templates || (n_spikes && (!grad_amplitude || !grad_shift)))
        return fail(FBP_E_ARG, "null gradient output");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const AdjArgs A = adj_args(dims, voltage, templates, spike_idx, spike_lab, amplitude, shift, n_spikes);
    const uint64_t nt = (uint64_t)A.M * A.C * A.W;
    FBP_CUDA(cudaMemsetAsync(grad_templates64, 0, nt * sizeof(double), st));
    if (n_spikes) {
        const size_t smem = (size_t)A.C * (A.W + 2) * sizeof(double);
        FBP_CUDA(allow_max_dyn_smem(adjoint_grad_kernel));
        count_launch();
        adjoint_grad_kernel<<<n_spikes < 148u * 16 ? n_spikes : 148u * 16, kAdjThreads, smem, st>>>(
            A, scale, grad_templates64, grad_amplitude, grad_shift);
    }
    count_launch();
    f64_to_f32_kernel<<<148 * 4, 256, 0, st>>>(grad_templates64, grad_templates, nt);
    FBP_CUDA(cudaGetLastError());
    return FBP_OK;
}
