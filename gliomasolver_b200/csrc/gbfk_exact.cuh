// Device arithmetic of the reference's RD operator, rounding for rounding.
//
// The reference evaluates ReactionDiffusionOperator<3>::operator()
// (Glioma/Operators/ReactionDiffusionOperator.h:97-138) with Real storage
// (float by default, double in the FP64 build) and double temporaries: h,
// ih2, the harmonic-mean quotient, the flux sums and the reaction term
// (:49-52,124-135, _harmonic_mean :148-163).  Every operation below is an
// explicitly rounded intrinsic (__fadd_rn, __dmul_rn, ...) so the compiler
// cannot contract a multiply and an add into an FMA, and the conversions
// between float and double happen exactly where C++'s usual arithmetic
// conversions put them in the reference.  The result is bit-identical to the
// reference's CPU build.
#pragma once
#include <cuda_runtime.h>

namespace gbfk {

__device__ __forceinline__ float radd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }

template <typename Real> __device__ __forceinline__ Real to_real(double x);
template <> __device__ __forceinline__ float to_real<float>(double x) { return __double2float_rn(x); }
template <> __device__ __forceinline__ double to_real<double>(double x) { return x; }

// df of a lab cell: p_w * Dw + p_g * Dg in Real (ReactionDiffusionOperator.h:105-111).
template <typename Real>
__device__ __forceinline__ Real diffusivity(Real pw, Real pg, Real Dw, Real Dg)
{
    return radd(rmul(pw, Dw), rmul(pg, Dg));
}

// Harmonic mean of a face, _harmonic_mean (ReactionDiffusionOperator.h:150-160):
//   df = (df + df_loc < eps) ? 0. : 2. * df * df_loc / (df + df_loc)
// with Real eps = 1e-8.  The value is symmetric in (df, df_loc): the float
// sum commutes, and 2*a*b is the same rounded double either way (2*a is
// exact and a*b commutes), so one evaluation serves both cells of a face.
template <typename Real>
__device__ __forceinline__ Real face_harmonic(Real df, Real df_loc)
{
    const Real eps = (Real)1.0e-08;
    const Real s = radd(df, df_loc);
    if (s < eps) return (Real)0.;
    const double num = __dmul_rn(__dmul_rn(2., (double)df), (double)df_loc);
    return to_real<Real>(__ddiv_rn(num, (double)s));
}

// Domain characteristic chf = phi + p_w + p_g (ReactionDiffusionOperator.h:115-120).
template <typename Real>
__device__ __forceinline__ Real domain_chf(Real phi, Real pw, Real pg)
{
    return radd(radd(phi, pw), pg);
}

// Right-hand side of one cell once the six face diffusivities df[0..5]
// (x-, x+, y-, y+, z-, z+, already harmonic-averaged) and the six
// neighbour chf values are known: _applyNoFluxBC (:166-181) and the flux
// sums (:125-135).  Returns dphidt in Real.
template <typename Real>
__device__ __forceinline__ Real cell_rhs(Real df0, Real df1, Real df2, Real df3, Real df4, Real df5,
                                         const Real chf[6], const Real phn[6], Real phi,
                                         Real rho, double ih2)
{
    const Real eps = (Real)0.1;
    if (chf[0] < eps) df1 = rmul(df1, (Real)2.0);
    if (chf[1] < eps) df0 = rmul(df0, (Real)2.0);
    if (chf[2] < eps) df3 = rmul(df3, (Real)2.0);
    if (chf[3] < eps) df2 = rmul(df2, (Real)2.0);
    if (chf[4] < eps) df5 = rmul(df5, (Real)2.0);
    if (chf[5] < eps) df4 = rmul(df4, (Real)2.0);

    Real sin_ = rmul(df0, phn[0]);
    sin_ = radd(sin_, rmul(df1, phn[1]));
    sin_ = radd(sin_, rmul(df2, phn[2]));
    sin_ = radd(sin_, rmul(df3, phn[3]));
    sin_ = radd(sin_, rmul(df4, phn[4]));
    sin_ = radd(sin_, rmul(df5, phn[5]));
    const double fluxIn = __dmul_rn(ih2, (double)sin_);

    Real sdf = radd(radd(radd(radd(radd(df0, df1), df2), df3), df4), df5);
    const double fluxOut = -__dmul_rn((double)rmul(sdf, phi), ih2);

    const double reaction = __dmul_rn((double)rmul(rho, phi), __dadd_rn(1., -(double)phi));
    return to_real<Real>(__dadd_rn(__dadd_rn(fluxOut, fluxIn), reaction));
}

// The same with the six no-flux tests already decided: low[k] is
// chf[k] < 0.1 of neighbour k (x-, x+, y-, y+, z-, z+).
template <typename Real>
__device__ __forceinline__ Real cell_rhs_flags(Real df0, Real df1, Real df2, Real df3, Real df4, Real df5,
                                               const bool low[6], const Real phn[6], Real phi, Real rho,
                                               double ih2)
{
    if (low[0]) df1 = rmul(df1, (Real)2.0);
    if (low[1]) df0 = rmul(df0, (Real)2.0);
    if (low[2]) df3 = rmul(df3, (Real)2.0);
    if (low[3]) df2 = rmul(df2, (Real)2.0);
    if (low[4]) df5 = rmul(df5, (Real)2.0);
    if (low[5]) df4 = rmul(df4, (Real)2.0);

    Real sin_ = rmul(df0, phn[0]);
    sin_ = radd(sin_, rmul(df1, phn[1]));
    sin_ = radd(sin_, rmul(df2, phn[2]));
    sin_ = radd(sin_, rmul(df3, phn[3]));
    sin_ = radd(sin_, rmul(df4, phn[4]));
    sin_ = radd(sin_, rmul(df5, phn[5]));
    const double fluxIn = __dmul_rn(ih2, (double)sin_);

    Real sdf = radd(radd(radd(radd(radd(df0, df1), df2), df3), df4), df5);
    const double fluxOut = -__dmul_rn((double)rmul(sdf, phi), ih2);

    const double reaction = __dmul_rn((double)rmul(rho, phi), __dadd_rn(1., -(double)phi));
    return to_real<Real>(__dadd_rn(__dadd_rn(fluxOut, fluxIn), reaction));
}

// UpdateTumor<3> (ReactionDiffusionOperator.h:219-221) with MRAG's max/min
// macros (MRAG/MRAGcore/MRAGCommon.h:19-37): phi += dt*dphidt; clamp to [0,1].
template <typename Real>
__device__ __forceinline__ Real cell_update(Real phi, Real dphidt, double dt)
{
    Real p = to_real<Real>(__dadd_rn((double)phi, __dmul_rn(dt, (double)dphidt)));
    p = ((Real)0. >= p) ? (Real)0. : p;
    p = ((Real)1. < p) ? (Real)1. : p;
    return p;
}

// The clamp of UpdateTumor alone: what the update leaves of phi when
// dphidt = 0 and dt is finite (phi + dt*0 rounds back to phi).
template <typename Real>
__device__ __forceinline__ Real clamp01(Real p)
{
    p = ((Real)0. >= p) ? (Real)0. : p;
    p = ((Real)1. < p) ? (Real)1. : p;
    return p;
}

// Inside-the-domain test p_w + p_g + phi > 0 (ReactionDiffusionOperator.h:103).
template <typename Real>
__device__ __forceinline__ bool in_domain(Real pw, Real pg, Real phi)
{
    return radd(radd(pw, pg), phi) > (Real)0.;
}

}  // namespace gbfk
