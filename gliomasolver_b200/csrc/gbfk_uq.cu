// The UQ end of the path: the finest-uniform dump of phi
// (Glioma_ReactionDiffusion::_dumpUQoutput, Glioma/Glioma_ReactionDiffusion.cpp:
// 208-262) and the log-likelihood of the observations
// (HGG_Likelihood.cpp:40-156 in tools/pi4u_lite/Inference/Likelihood/source),
// both on the device so that a TMCMC sample never leaves HBM.
#include "gbfk_exact.cuh"
#include "gbfk_kernels.cuh"

namespace gbfk {

// One thread per pool cell.  x = origin + h*i in Real (BlockInfo::pos,
// MRAG/MRAGcore/MRAGCommon.h:199), voxel m = floor(x / hf).  Blocks at least as
// fine as the dump grid write their voxel from the last cell that maps to it in
// the reference's z, y, x loop order; coarser blocks write c^3 copies with
// c = 2, 3 or 4 chosen by h exactly as the reference does.
template <typename Real>
__global__ void uq_dump_kernel(const int *__restrict__ slot, const Real *__restrict__ origin,
                               const Real *__restrict__ hblk, int nblocks, const Real *__restrict__ phi, int gpd,
                               double *__restrict__ out)
{
    const int64_t n = (int64_t)nblocks * kBS3;
    const double hf = 1. / gpd;
    const double eps = hf * 0.5;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i >> 9), c = (int)(i & 511);
        const int ix = c & 7, iy = (c >> 3) & 7, iz = c >> 6;
        const Real hb = hblk[b];
        const Real o0 = origin[3 * b], o1 = origin[3 * b + 1], o2 = origin[3 * b + 2];
        const double x0 = radd(o0, rmul(hb, (Real)ix)), x1 = radd(o1, rmul(hb, (Real)iy)),
                     x2 = radd(o2, rmul(hb, (Real)iz));
        const int mx = (int)floor(__ddiv_rn(x0, hf)), my = (int)floor(__ddiv_rn(x1, hf)),
                  mz = (int)floor(__ddiv_rn(x2, hf));
        const double hd = hb;
        const double v = (double)phi[(int64_t)slot[b] * kBS3 + c];
        int cc;
        if (hd < hf + eps) {
            // last writer of the voxel in loop order: the next cell along each
            // direction maps to another voxel or lies outside the block
            const bool lx = ix == 7 || (int)floor(__ddiv_rn((double)radd(o0, rmul(hb, (Real)(ix + 1))), hf)) != mx;
            const bool ly = iy == 7 || (int)floor(__ddiv_rn((double)radd(o1, rmul(hb, (Real)(iy + 1))), hf)) != my;
            const bool lz = iz == 7 || (int)floor(__ddiv_rn((double)radd(o2, rmul(hb, (Real)(iz + 1))), hf)) != mz;
            if (!(lx && ly && lz)) continue;
            cc = 1;
        } else if (hd < 2. * hf + eps) cc = 2;
        else if (hd < 3. * hf + eps) cc = 3;
        else cc = 4;
        for (int cz = 0; cz < cc; cz++)
            for (int cy = 0; cy < cc; cy++)
                for (int cx = 0; cx < cc; cx++)
                    out[(mx + cx) + (int64_t)gpd * ((my + cy) + (int64_t)gpd * (mz + cz))] = v;
    }
}

template <typename Real>
cudaError_t launch_uq_dump(const int *slot, const Real *origin, const Real *hblk, int nblocks, const Real *phi,
                           int gpd, double *out, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (size_t)gpd * gpd * gpd, s);
    if (e != cudaSuccess || nblocks <= 0) return e;
    int64_t nb = ((int64_t)nblocks * kBS3 + 255) / 256;
    if (nb > 148 * 32) nb = 148 * 32;
    uq_dump_kernel<Real><<<(int)nb, 256, 0, s>>>(slot, origin, hblk, nblocks, phi, gpd, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Log-likelihood terms with compensated (Neumaier) double sums.  The
// reference sums in long double; with compensation the device sums carry
// about 106 bits, and each term is the exact value of the reference's
// expression computed without cancellation:
//   alpha = 0.5 + 0.5*sgn(d)*(1 - exp(-t)),  t = omega2/slope,
//   omega2 = 1 if d > 0 else d^2,  d = u - uc       (HGG_Likelihood.cpp:149-155)
// so for d > 0: log(alpha) = log1p(-e/2), log(1-alpha) = log(1/2) - t,
//    for d < 0: log(alpha) = log(1/2) - t, log(1-alpha) = log1p(-e/2), e = exp(-t).
struct Neumaier {
    double s, c;
    __device__ void add(double x)
    {
        const double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    __device__ void merge(const Neumaier &o)
    {
        add(o.s);
        add(o.c);
    }
};

__device__ __forceinline__ void bernoulli_terms(double u, double uc, double is2, double &log_a, double &log_1a)
{
    const double d = u - uc;
    const int sg = (d < -0.0) ? -1 : (d > 0.0 ? 1 : 0);
    const double t = (d > 0.) ? is2 : d * d * is2;
    const double lhalf = -0.69314718055994530942;  // log(1/2)
    if (sg == 0) {
        log_a = log_1a = lhalf;
    } else {
        const double e = exp(-t);
        const double a = log1p(-0.5 * e), b = lhalf - t;
        log_a = sg > 0 ? a : b;
        log_1a = sg > 0 ? b : a;
    }
}

constexpr int kLikThreads = 256;

__global__ void __launch_bounds__(kLikThreads)
likelihood_partial_kernel(const double *__restrict__ model, int n, const unsigned char *__restrict__ t1c,
                          const unsigned char *__restrict__ flair, const double *__restrict__ pet,
                          const int *__restrict__ roi, int nroi, LikelihoodParams p, double *__restrict__ partial)
{
    Neumaier spet = {0, 0}, st1 = {0, 0}, st2 = {0, 0};
    double npet = 0;
    const int64_t N = (int64_t)n * n * n;
    const double is2 = 1. / p.slope;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (pet) {
        for (int64_t g = i0; g < N; g += stride) {
            const int ix = (int)(g % n), iy = (int)((g / n) % n), iz = (int)(g / ((int64_t)n * n));
            if (ix % p.step_pet == 0 && iy % p.step_pet == 0 && iz % p.step_pet == 0 && pet[g] > 0.) {
                const double r = model[g] - p.pet_scale * pet[g];
                spet.add(r * r);
                npet += 1;
            }
        }
    }
    if (!roi) {
        for (int64_t g = i0; g < N; g += stride) {
            double a, b;
            bernoulli_terms(model[g], p.t1_uc, is2, a, b);
            st1.add(t1c[g] ? a : b);
            bernoulli_terms(model[g], p.t2_uc, is2, a, b);
            st2.add(flair[g] ? a : b);
        }
    } else {
        for (int64_t k = i0; k < nroi; k += stride) {
            const int ix = roi[3 * k], iy = roi[3 * k + 1], iz = roi[3 * k + 2];
            if (ix % p.step_mri != 0 || iy % p.step_mri != 0 || iz % p.step_mri != 0) continue;
            const int64_t g = ix + (int64_t)n * (iy + (int64_t)n * iz);
            double a, b;
            bernoulli_terms(model[g], p.t1_uc, is2, a, b);
            st1.add(t1c[g] ? a : b);
            bernoulli_terms(model[g], p.t2_uc, is2, a, b);
            st2.add(flair[g] ? a : b);
        }
    }
    // deterministic tree reduction inside the CTA
    __shared__ double red[7][kLikThreads];
    const int t = threadIdx.x;
    red[0][t] = spet.s; red[1][t] = spet.c; red[2][t] = npet;
    red[3][t] = st1.s; red[4][t] = st1.c; red[5][t] = st2.s; red[6][t] = st2.c;
    __syncthreads();
    for (int w = kLikThreads / 2; w > 0; w >>= 1) {
        if (t < w) {
            Neumaier a = {red[0][t], red[1][t]}, b = {red[0][t + w], red[1][t + w]};
            a.merge(b);
            red[0][t] = a.s; red[1][t] = a.c;
            red[2][t] += red[2][t + w];
            Neumaier c1 = {red[3][t], red[4][t]}, d1 = {red[3][t + w], red[4][t + w]};
            c1.merge(d1);
            red[3][t] = c1.s; red[4][t] = c1.c;
            Neumaier c2 = {red[5][t], red[6][t]}, d2 = {red[5][t + w], red[6][t + w]};
            c2.merge(d2);
            red[5][t] = c2.s; red[6][t] = c2.c;
        }
        __syncthreads();
    }
    if (t < 7) partial[blockIdx.x * 7 + t] = red[t][0];
}

__global__ void likelihood_final_kernel(const double *__restrict__ partial, int nparts, int have_pet,
                                        LikelihoodParams p, double *__restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Neumaier spet = {0, 0}, st1 = {0, 0}, st2 = {0, 0};
    double npet = 0;
    for (int i = 0; i < nparts; i++) {
        const double *q = partial + 7 * i;
        Neumaier a = {q[0], q[1]}, b = {q[3], q[4]}, c = {q[5], q[6]};
        spet.merge(a);
        npet += q[2];
        st1.merge(b);
        st2.merge(c);
    }
    const double PI = 3.14159265358979323846;
    double lpet = 0;
    if (have_pet) {
        const double p1 = -0.5 * npet * log(2. * PI * p.pet_sigma2);
        const double p2 = -0.5 * (1. / p.pet_sigma2) * (spet.s + spet.c);
        lpet = p1 + p2;
    }
    out[0] = lpet;
    out[1] = st1.s + st1.c;
    out[2] = st2.s + st2.c;
    out[3] = out[0] + out[1] + out[2];
}

cudaError_t launch_likelihood(const double *model, int n, const unsigned char *t1c, const unsigned char *flair,
                              const double *pet, const int *roi, int nroi, const LikelihoodParams &p,
                              double *partial, int nparts, double *out, cudaStream_t s)
{
    likelihood_partial_kernel<<<nparts, kLikThreads, 0, s>>>(model, n, t1c, flair, pet, roi, nroi, p, partial);
    likelihood_final_kernel<<<1, 32, 0, s>>>(partial, nparts, pet != nullptr, p, out);
    return cudaGetLastError();
}

template cudaError_t launch_uq_dump<float>(const int *, const float *, const float *, int, const float *, int,
                                           double *, cudaStream_t);
template cudaError_t launch_uq_dump<double>(const int *, const double *, const double *, int, const double *, int,
                                            double *, cudaStream_t);

}  // namespace gbfk
