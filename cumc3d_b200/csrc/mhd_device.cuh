// mhd_device.cuh -- per-face / per-cell arithmetic of the MHD stage, device side.
//
// Every function here restates one routine of the reference
// (leon-astrophy/cumc3d, solver/mhd/*.f90) with the SAME floating-point
// operation order as the Fortran source (left-to-right, x**2 -> x*x).  The
// FP64 translation unit is compiled with --fmad=false so that these functions
// produce the same bits as the Fortran semantics; the FP32 unit instantiates
// the same templates with T = float.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cumc {

// variable indices (solver/mhd/setup.f90:39-96), 1-based as in the reference
enum : int { irho = 1, ivx = 2, ivy = 3, ivz = 4, itau = 5, ibx = 6, iby = 7, ibz = 8 };
// face-EMF slots (solver/mhd/mhd_module.f90:19-24), 0-based here
enum : int { e_yx = 0, e_zx = 1, e_xy = 2, e_zy = 3, e_xz = 4, e_yz = 5 };

enum : int { REC_TVD_MM = 0, REC_TVD_VL = 1, REC_TVD_MC = 2, REC_PPM = 3, REC_WENO = 4 };
enum : int { RS_LF = 0, RS_HLL = 1, RS_HLLC = 2, RS_HLLD = 3 };

template <class T> __device__ __forceinline__ T dsqrt(T x);
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <class T> __device__ __forceinline__ T dabs(T x);
template <> __device__ __forceinline__ double dabs<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float dabs<float>(float x) { return fabsf(x); }
// x / y bit for bit, minus the FP64 division's slow path for x == 0 (a
// zero numerator is common: fluid at rest, zero field components, flat
// stencils).  For x == +-0 and a normal y the quotient of a stand-in
// numerator (chosen in inline PTX, so the optimizer cannot put x back) is
// discarded and the signed zero sign(x) * sign(y) returned; every other case
// is the ordinary division.  The tests run on the integer pipe, which the
// FP64-bound kernels leave idle, on the 32-bit words of the operands (one
// logic op and one compare per test).  FP32 divides directly.
template <class T> __device__ __forceinline__ T dv(T x, T y) { return x / y; }
template <> __device__ __forceinline__ double dv<double>(double x, double y) {
    const unsigned xh = (unsigned)__double2hiint(x), xl = (unsigned)__double2loint(x);
    const unsigned yh = (unsigned)__double2hiint(y);
    // x == +-0: no bit set but the sign; y normal: biased exponent 1..2046
    const int z = (((xh & 0x7FFFFFFFu) | xl) == 0u) & (((yh & 0x7FF00000u) - 0x00100000u) < 0x7FE00000u);
    unsigned nh, nl;
    asm("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\tselp.b32 %0, 0x3FF00000, %2, p;\n\tselp.b32 %1, 0, %3, p;\n\t}"
        : "=r"(nh), "=r"(nl)
        : "r"(xh), "r"(xl), "r"(z));
    const double q = __hiloint2double((int)nh, (int)nl) / y;
    const double zr = __hiloint2double((int)((xh ^ yh) & 0x80000000u), 0);
    return z ? zr : q;
}

// Fortran SIGN(1, x)
template <class T> __device__ __forceinline__ T sign1(T x);
template <> __device__ __forceinline__ double sign1<double>(double x) { return copysign(1.0, x); }
template <> __device__ __forceinline__ float sign1<float>(float x) { return copysignf(1.0f, x); }
// min/max with the comparison the oracle uses: (b < a) ? b : a
template <class T> __device__ __forceinline__ T dmin(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T dmax(T a, T b) { return (b > a) ? b : a; }
template <class T> __device__ __forceinline__ T dmin3(T a, T b, T c) { return dmin(dmin(a, b), c); }
template <class T> __device__ __forceinline__ T dmax3(T a, T b, T c) { return dmax(dmax(a, b), c); }

// ---------------------------------------------------------------------------
// reconstruction kernels on one cell (vm_out = left edge, vp_out = right edge)
// ---------------------------------------------------------------------------

// PPMC, solver/mhd/ppmc_module.f90:359-464 (Colella-Woodward, no steepening)
template <class T>
__device__ __forceinline__ void ppmc(const T *__restrict__ w, T vm2, T vm1, T vc, T vp1, T vp2, T &vm_out, T &vp_out) {
    const T a0m = w[0], a1m = w[1], a2m = w[2], a3m = w[3];
    const T a0p = w[4], a1p = w[5], a2p = w[6], a3p = w[7];
    const T b0m = w[8], b1m = w[9], b0c = w[10], b1c = w[11], b0p = w[12], b1p = w[13];
    T deltap1 = b0p * (vp2 - vp1) + b1p * (vp1 - vc);
    T deltac = b0c * (vp1 - vc) + b1c * (vc - vm1);
    T deltam1 = b0m * (vc - vm1) + b1m * (vm1 - vm2);
    T dmc, dmp1, dmm1, condition;
    condition = (vp1 - vc) * (vc - vm1);
    if (condition > T(0)) dmc = dmin3(dabs(deltac), T(2) * dabs(vc - vm1), T(2) * dabs(vc - vp1)) * sign1(deltac);
    else dmc = T(0);
    condition = (vp2 - vp1) * (vp1 - vc);
    if (condition > T(0)) dmp1 = dmin3(dabs(deltap1), T(2) * dabs(vp1 - vc), T(2) * dabs(vp1 - vp2)) * sign1(deltap1);
    else dmp1 = T(0);
    condition = (vc - vm1) * (vm1 - vm2);
    if (condition > T(0)) dmm1 = dmin3(dabs(deltam1), T(2) * dabs(vm1 - vm2), T(2) * dabs(vm1 - vc)) * sign1(deltam1);
    else dmm1 = T(0);
    vp_out = vc + a0p * (vp1 - vc) + a1p * (vp1 - vc) + a2p * dmp1 + a3p * dmc;
    vm_out = vm1 + a0m * (vc - vm1) + a1m * (vc - vm1) + a2m * dmc + a3m * dmm1;
    const T vl = vm_out, vr = vp_out;
    if ((vr - vc) * (vc - vl) <= T(0)) {
        vp_out = vc;
        vm_out = vc;
    } else {
        condition = (vr - vl) * (vl - T(3) * vc + T(2) * vr);
        if (condition < T(0)) vm_out = T(3) * vc - T(2) * vr;
        condition = (vp_out - vm_out) * (T(3) * vc - T(2) * vl - vr);
        if (condition < T(0)) vp_out = T(3) * vc - T(2) * vl;
    }
}

// WENO-Z, solver/mhd/weno_module.f90:315-408 (tau5 = |beta1 - beta3|, eps = 1e-40)
// epsilon of the WENO-Z weights: the reference's 1e-40 in FP64; the FP32 form
// uses 1e-30 (1e-40 is subnormal in FP32) and caps the ratio so its square
// stays finite
template <class T> struct WenoEps;
template <> struct WenoEps<double> {
    static __device__ __forceinline__ double eps() { return 1.0e-40; }
    static __device__ __forceinline__ double cap(double q) { return q; }
};
template <> struct WenoEps<float> {
    static __device__ __forceinline__ float eps() { return 1.0e-30f; }
    static __device__ __forceinline__ float cap(float q) { return fminf(q, 1.0e15f); }
};

template <class T>
__device__ __forceinline__ T wenoz_combine(T P1, T P2, T P3, T B1, T B2, T B3) {
    const T smallpara = WenoEps<T>::eps();
    const T g1 = T(1.0 / 10.0), g2 = T(6.0 / 10.0), g3 = T(3.0 / 10.0);
    T tau5 = dabs(B1 - B3);
    T q1 = WenoEps<T>::cap(dv(tau5, smallpara + B1)), q2 = WenoEps<T>::cap(dv(tau5, smallpara + B2)),
      q3 = WenoEps<T>::cap(dv(tau5, smallpara + B3));
    T w1 = g1 * (T(1) + q1 * q1);
    T w2 = g2 * (T(1) + q2 * q2);
    T w3 = g3 * (T(1) + q3 * q3);
    return dv(w1 * P1 + w2 * P2 + w3 * P3, w1 + w2 + w3);
}

// x / 3 rounded to nearest.  FP64: the quotient q = RN(x * RN(1/3)) is within
// one ulp of x/3, the remainder x - 3q is exact with one FMA, and one more FMA
// q + r * RN(1/3) rounds to the correctly rounded quotient (Markstein's
// correction; x/3 is never a rounding midpoint since 3m would need p+1 bits).
// The result equals the IEEE division bit for bit (checked on 2^30+ inputs by
// tests/test_numerics_gpu.py) at a fraction of its cost.
template <class T> __device__ __forceinline__ T div3(T x);
template <> __device__ __forceinline__ double div3<double>(double x) {
    const double z = 1.0 / 3.0;
    const double q = __dmul_rn(x, z);
    const double r = __fma_rn(-q, 3.0, x);
    return __fma_rn(r, z, q);
}
template <> __device__ __forceinline__ float div3<float>(float x) { return x * (1.0f / 3.0f); }

template <class T>
__device__ __forceinline__ void weno(const T *__restrict__ w, T vm2, T vm1, T vc, T vp1, T vp2, T &vm_out, T &vp_out) {
    const T r1 = T(13.0 / 12.0), r2 = T(1.0 / 4.0);
    T U01 = w[0] * vc + w[1] * vp1;
    T U12 = w[2] * vp1 + w[3] * vp2;
    T U10 = w[4] * vm1 + w[5] * vc;
    T U21 = w[6] * vm2 + w[7] * vm1;
    T U00 = vm1 + w[8] * (vm1 - vm2);
    T U11 = vp1 + w[9] * (vp1 - vp2);
    {
        T P1 = div3(T(6) * vc - T(1) * U10 - T(2) * U00);
        T P2 = div3(-T(1) * U10 + T(2) * vc + T(2) * U01);
        T P3 = div3(T(2) * U01 + T(2) * vp1 - T(1) * U12);
        T t1 = T(2) * U10 - T(2) * U00, t2 = T(4) * vc - T(2) * U10 - T(2) * U00;
        T B1 = r1 * (t1 * t1) + r2 * (t2 * t2);
        T t3 = T(2) * U10 - T(4) * vc + T(2) * U01, t4 = -T(2) * U10 + T(2) * U01;
        T B2 = r1 * (t3 * t3) + r2 * (t4 * t4);
        T t5 = T(2) * U01 - T(4) * vp1 + T(2) * U12, t6 = -T(6) * U01 + T(8) * vp1 - T(2) * U12;
        T B3 = r1 * (t5 * t5) + r2 * (t6 * t6);
        vp_out = wenoz_combine(P1, P2, P3, B1, B2, B3);
    }
    {
        T P1 = div3(T(6) * vc - T(1) * U01 - T(2) * U11);
        T P2 = div3(-T(1) * U01 + T(2) * vc + T(2) * U10);
        T P3 = div3(T(2) * U10 + T(2) * vm1 - T(1) * U21);
        T t1 = T(2) * U01 - T(2) * U11, t2 = T(4) * vc - T(2) * U01 - T(2) * U11;
        T B1 = r1 * (t1 * t1) + r2 * (t2 * t2);
        T t3 = T(2) * U01 - T(4) * vc + T(2) * U10, t4 = T(2) * U01 - T(2) * U10;
        T B2 = r1 * (t3 * t3) + r2 * (t4 * t4);
        T t5 = T(2) * U10 - T(4) * vm1 + T(2) * U21, t6 = T(8) * vm1 - T(6) * U10 - T(2) * U21;
        T B3 = r1 * (t5 * t5) + r2 * (t6 * t6);
        vm_out = wenoz_combine(P1, P2, P3, B1, B2, B3);
    }
}

// The pieces of weno() above, for the learned smooth-face path: candidate
// values P and smoothness indicators B of the right (p) and left (m) faces,
// with the same expressions in the same order.
template <class T> struct WenoParts { T Pp[3], Bp[3], Pm[3], Bm[3]; };
template <class T>
__device__ __forceinline__ void weno_parts(const T *__restrict__ w, T vm2, T vm1, T vc, T vp1, T vp2, WenoParts<T> &o) {
    const T r1 = T(13.0 / 12.0), r2 = T(1.0 / 4.0);
    T U01 = w[0] * vc + w[1] * vp1;
    T U12 = w[2] * vp1 + w[3] * vp2;
    T U10 = w[4] * vm1 + w[5] * vc;
    T U21 = w[6] * vm2 + w[7] * vm1;
    T U00 = vm1 + w[8] * (vm1 - vm2);
    T U11 = vp1 + w[9] * (vp1 - vp2);
    o.Pp[0] = div3(T(6) * vc - T(1) * U10 - T(2) * U00);
    o.Pp[1] = div3(-T(1) * U10 + T(2) * vc + T(2) * U01);
    o.Pp[2] = div3(T(2) * U01 + T(2) * vp1 - T(1) * U12);
    {
        T t1 = T(2) * U10 - T(2) * U00, t2 = T(4) * vc - T(2) * U10 - T(2) * U00;
        o.Bp[0] = r1 * (t1 * t1) + r2 * (t2 * t2);
        T t3 = T(2) * U10 - T(4) * vc + T(2) * U01, t4 = -T(2) * U10 + T(2) * U01;
        o.Bp[1] = r1 * (t3 * t3) + r2 * (t4 * t4);
        T t5 = T(2) * U01 - T(4) * vp1 + T(2) * U12, t6 = -T(6) * U01 + T(8) * vp1 - T(2) * U12;
        o.Bp[2] = r1 * (t5 * t5) + r2 * (t6 * t6);
    }
    o.Pm[0] = div3(T(6) * vc - T(1) * U01 - T(2) * U11);
    o.Pm[1] = div3(-T(1) * U01 + T(2) * vc + T(2) * U10);
    o.Pm[2] = div3(T(2) * U10 + T(2) * vm1 - T(1) * U21);
    {
        T t1 = T(2) * U01 - T(2) * U11, t2 = T(4) * vc - T(2) * U01 - T(2) * U11;
        o.Bm[0] = r1 * (t1 * t1) + r2 * (t2 * t2);
        T t3 = T(2) * U01 - T(4) * vc + T(2) * U10, t4 = T(2) * U01 - T(2) * U10;
        o.Bm[1] = r1 * (t3 * t3) + r2 * (t4 * t4);
        T t5 = T(2) * U10 - T(4) * vm1 + T(2) * U21, t6 = T(8) * vm1 - T(6) * U10 - T(2) * U21;
        o.Bm[2] = r1 * (t5 * t5) + r2 * (t6 * t6);
    }
}

// linear (optimal-weight) fifth-order face values: the WENO candidates
// combined with g = (0.1, 0.6, 0.3) instead of the nonlinear weights
template <class T>
__device__ __forceinline__ void weno_linear(const T *__restrict__ w, T vm2, T vm1, T vc, T vp1, T vp2, T &vm_out,
                                            T &vp_out) {
    T U01 = w[0] * vc + w[1] * vp1;
    T U12 = w[2] * vp1 + w[3] * vp2;
    T U10 = w[4] * vm1 + w[5] * vc;
    T U21 = w[6] * vm2 + w[7] * vm1;
    T U00 = vm1 + w[8] * (vm1 - vm2);
    T U11 = vp1 + w[9] * (vp1 - vp2);
    const T g1 = T(1.0 / 10.0), g2 = T(6.0 / 10.0), g3 = T(3.0 / 10.0);
    vp_out = g1 * div3(T(6) * vc - T(1) * U10 - T(2) * U00) + g2 * div3(-T(1) * U10 + T(2) * vc + T(2) * U01) +
             g3 * div3(T(2) * U01 + T(2) * vp1 - T(1) * U12);
    vm_out = g1 * div3(T(6) * vc - T(1) * U01 - T(2) * U11) + g2 * div3(-T(1) * U01 + T(2) * vc + T(2) * U10) +
             g3 * div3(T(2) * U10 + T(2) * vm1 - T(1) * U21);
}

// normalised WENO-Z weights (the ones wenoz_combine applies)
template <class T>
__device__ __forceinline__ void wenoz_weights(const T B[3], T om[3]) {
    const T smallpara = WenoEps<T>::eps();
    const T g1 = T(1.0 / 10.0), g2 = T(6.0 / 10.0), g3 = T(3.0 / 10.0);
    T tau5 = dabs(B[0] - B[2]);
    T q1 = WenoEps<T>::cap(dv(tau5, smallpara + B[0])), q2 = WenoEps<T>::cap(dv(tau5, smallpara + B[1])),
      q3 = WenoEps<T>::cap(dv(tau5, smallpara + B[2]));
    T w1 = g1 * (T(1) + q1 * q1);
    T w2 = g2 * (T(1) + q2 * q2);
    T w3 = g3 * (T(1) + q3 * q3);
    T sum = w1 + w2 + w3;
    om[0] = w1 / sum;
    om[1] = w2 / sum;
    om[2] = w3 / sum;
}

// TVD (Mignone 2014) limiters, solver/mhd/tvd_module.f90:279-344
template <class T, int LIM>
__device__ __forceinline__ void tvd(const T *__restrict__ w, T vm, T vc, T vp, T &vm_out, T &vp_out) {
    const T cf = w[0], cb = w[1];
    T dqf = dv(T(2) * (vp - vc), cf);
    T dqb = dv(T(2) * (vc - vm), cb);
    T slope;
    if (LIM == REC_TVD_MM) {
        slope = T(0.5) * (sign1(dqf) + sign1(dqb)) * dmin(dabs(dqf), dabs(dqb));
    } else if (LIM == REC_TVD_VL) {
        T dq2 = dqf * dqb;
        if (dq2 <= T(0)) slope = T(0);
        else slope = dv(dq2 * (cf * dqb + cb * dqf), dqb * dqb + dqf * dqf + dq2 * (cf + cb - T(2)));
    } else {
        if (dqf == T(0)) slope = T(0);
        else {
            T v_tvd = dv(dqb, dqf);
            slope = dmax(T(0), dmin3(T(0.5) * (T(1) + v_tvd), cf, cb * v_tvd));
            slope = dqf * slope;
        }
    }
    vp_out = vc + T(0.5) * slope;
    vm_out = vc - T(0.5) * slope;
}

template <class T, int REC>
__device__ __forceinline__ void recon_cell(const T *__restrict__ w, T vm2, T vm1, T vc, T vp1, T vp2, T &vm_out, T &vp_out) {
    if (REC == REC_PPM) ppmc<T>(w, vm2, vm1, vc, vp1, vp2, vm_out, vp_out);
    else if (REC == REC_WENO) weno<T>(w, vm2, vm1, vc, vp1, vp2, vm_out, vp_out);
    else tvd<T, REC>(w, vm1, vc, vp1, vm_out, vp_out);
}

// ---------------------------------------------------------------------------
// Riemann solvers, solver/mhd/rsolver_module.f90
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T signalspeed(T cs, T bn, T bt1, T bt2, T rho) {  // 32-48
    T a2 = cs * cs;
    T a4 = a2 * a2;
    T b2n = dv(bn * bn, rho);
    T b2t1 = dv(bt1 * bt1, rho);
    T b2t2 = dv(bt2 * bt2, rho);
    T b2 = b2n + b2t1 + b2t2;
    T b4 = b2 * b2;
    return dsqrt(T(0.5) * (a2 + b2 + dsqrt(dmax((a4 + b4 + T(2) * b2 * a2) - T(4) * a2 * b2n, T(0)))));
}
template <class T> __device__ __forceinline__ T hll_state(T ul, T ur, T fl, T fr, T sl, T sr) {  // 54-59
    return dv(sr * ur - sl * ul - (fr - fl), sr - sl);
}
template <class T> __device__ __forceinline__ T hll_flux(T yl, T yr, T xl, T xr, T sl, T sr) {  // 61-66
    return dv(sr * yl - sl * yr + sl * sr * (xr - xl), sr - sl);
}
template <class T> __device__ __forceinline__ T roe_avg(T xl, T xr, T rhol, T rhor) {  // 68-73
    return dv(dsqrt(rhol) * xl + dsqrt(rhor) * xr, dsqrt(rhol) + dsqrt(rhor));
}
template <class T>
__device__ __forceinline__ T sstar_hllc(T pl, T pr, T rhol, T rhor, T vl, T vr, T sl, T sr, T bl, T br) {  // 86-93
    return dv(rhor * vr * (sr - vr) - rhol * vl * (sl - vl) + pl - pr + br * br - bl * bl, rhor * (sr - vr) - rhol * (sl - vl));
}

// direction -> (normal, transverse) component indices, BUILDSTATES spatial.f90:306-331
template <int DIR> struct Frame;
template <> struct Frame<0> { static constexpr int ivn = ivx, ivt1 = ivy, ivt2 = ivz, ibn = ibx, ibt1 = iby, ibt2 = ibz; };
template <> struct Frame<1> { static constexpr int ivn = ivy, ivt1 = ivz, ivt2 = ivx, ibn = iby, ibt1 = ibz, ibt2 = ibx; };
template <> struct Frame<2> { static constexpr int ivn = ivz, ivt1 = ivx, ivt2 = ivy, ibn = ibz, ibt1 = ibx, ibt2 = iby; };

// BUILDSTATES (spatial.f90:336-392) for one side of one face.
// p[1..8] primitive face state; u, f outputs (1-based, index 0 unused).
template <class T, int DIR>
__device__ __forceinline__ void build_state(const T *p, T eps, T *u, T *f) {
    using F = Frame<DIR>;
    T b2 = p[ibx] * p[ibx] + p[iby] * p[iby] + p[ibz] * p[ibz];
    T v2 = p[ivx] * p[ivx] + p[ivy] * p[ivy] + p[ivz] * p[ivz];
    T vb = p[ibx] * p[ivx] + p[iby] * p[ivy] + p[ibz] * p[ivz];
    u[irho] = p[irho];
    u[ivx] = p[ivx] * p[irho];
    u[ivy] = p[ivy] * p[irho];
    u[ivz] = p[ivz] * p[irho];
    u[ibx] = p[ibx];
    u[iby] = p[iby];
    u[ibz] = p[ibz];
    u[itau] = p[irho] * (T(0.5) * v2 + eps) + T(0.5) * b2;
#pragma unroll
    for (int i = irho; i <= itau; ++i) f[i] = u[i] * p[F::ivn];
    f[F::ivn] = f[F::ivn] + p[itau] + T(0.5) * (b2) - p[F::ibn] * p[F::ibn];
    f[F::ivt1] = f[F::ivt1] - p[F::ibn] * p[F::ibt1];
    f[F::ivt2] = f[F::ivt2] - p[F::ibn] * p[F::ibt2];
    f[itau] = f[itau] + (p[itau] + T(0.5) * (b2)) * p[F::ivn] - p[F::ibn] * vb;
    f[F::ibn] = T(0);
    f[F::ibt1] = (p[F::ivn] * p[F::ibt1] - p[F::ivt1] * p[F::ibn]);
    f[F::ibt2] = (p[F::ivn] * p[F::ibt2] - p[F::ivt2] * p[F::ibn]);
}

// HLLC star region, rsolver_module.f90:423-498
template <class T, int DIR>
__device__ __forceinline__ void hllc_star(const T *pl, const T *pr, const T *ul, const T *ur, const T *fl, const T *fr,
                                          T *fo, T sL, T sR, T pLt, T pRt) {
    using F = Frame<DIR>;
    constexpr int ivn = F::ivn, ivt1 = F::ivt1, ivt2 = F::ivt2, ibn = F::ibn, ibt1 = F::ibt1, ibt2 = F::ibt2;
    T u_hll[9], p_hll[9], us[9];
    T sstar = sstar_hllc(pLt, pRt, pl[irho], pr[irho], pl[ivn], pr[ivn], sL, sR, pl[ibn], pr[ibn]);
    u_hll[ibn] = pl[ibn];
    u_hll[ibt1] = hll_state(pl[ibt1], pr[ibt1], fl[ibt1], fr[ibt1], sL, sR);
    u_hll[ibt2] = hll_state(pl[ibt2], pr[ibt2], fl[ibt2], fr[ibt2], sL, sR);
    u_hll[irho] = hll_state(pl[irho], pr[irho], fl[irho], fr[irho], sL, sR);
    u_hll[ivt1] = hll_state(ul[ivt1], ur[ivt1], fl[ivt1], fr[ivt1], sL, sR);
    u_hll[ivt2] = hll_state(ul[ivt2], ur[ivt2], fl[ivt2], fr[ivt2], sL, sR);
    p_hll[ivn] = sstar;
    p_hll[ivt1] = dv(u_hll[ivt1], u_hll[irho]);
    p_hll[ivt2] = dv(u_hll[ivt2], u_hll[irho]);
    const bool left = (sstar >= T(0));
    const T *pS = left ? pl : pr;
    const T *uS = left ? ul : ur;
    const T *fS = left ? fl : fr;
    const T s = left ? sL : sR, pSt = left ? pLt : pRt;
    us[irho] = dv(uS[irho] * (s - pS[ivn]), s - sstar);
    T vb = pS[ibx] * pS[ivx] + pS[iby] * pS[ivy] + pS[ibz] * pS[ivz];
    T vbhll = u_hll[ibx] * p_hll[ivx] + u_hll[iby] * p_hll[ivy] + u_hll[ibz] * p_hll[ivz];
    T ps = pS[irho] * (s - pS[ivn]) * (sstar - pS[ivn]) + pSt;
    us[ibn] = u_hll[ibn];
    us[ibt1] = u_hll[ibt1];
    us[ibt2] = u_hll[ibt2];
    us[ivn] = us[irho] * sstar;
    us[ivt1] = dv(uS[ivt1] * (s - pS[ivn]) - (us[ibn] * us[ibt1] - pS[ibn] * pS[ibt1]), s - sstar);
    us[ivt2] = dv(uS[ivt2] * (s - pS[ivn]) - (us[ibn] * us[ibt2] - pS[ibn] * pS[ibt2]), s - sstar);
    us[itau] = dv(uS[itau] * (s - pS[ivn]) + (ps * sstar - pSt * pS[ivn]) - ((vbhll * us[ibn] - vb * pS[ibn])), s - sstar);
#pragma unroll
    for (int i = 1; i <= 8; ++i) fo[i] = fS[i] + s * (us[i] - uS[i]);
}

// HLLD star / double-star regions, rsolver_module.f90:613-750.  The normal
// component of the double-star states (never assigned in the reference) is
// the constant normal field B_n.
template <class T, int DIR>
__device__ __forceinline__ void hlld_star(const T *pl, const T *pr, const T *ul, const T *ur, const T *fl, const T *fr,
                                          T *fo, T sL, T sR, T pLt, T pRt) {
    using F = Frame<DIR>;
    constexpr int ivn = F::ivn, ivt1 = F::ivt1, ivt2 = F::ivt2, ibn = F::ibn, ibt1 = F::ibt1, ibt2 = F::ibt2;
    T usL[9], usR[9], pstL[9], pstR[9];
    T sM = sstar_hllc(pLt, pRt, pl[irho], pr[irho], pl[ivn], pr[ivn], sL, sR, pl[ibn], pr[ibn]);
#pragma unroll
    for (int i = irho; i <= itau; ++i) usL[i] = dv(ul[i] * (sL - pl[ivn]), sL - sM);
#pragma unroll
    for (int i = irho; i <= itau; ++i) usR[i] = dv(ur[i] * (sR - pr[ivn]), sR - sM);
    T sstarL = sM - dv(dabs(pl[ibn]), dsqrt(usL[irho]));
    T sstarR = sM + dv(dabs(pr[ibn]), dsqrt(usR[irho]));
    if (((sstarL - sL) < T(1.0e-4) * (sM - sL)) || ((sstarR - sR) > -T(1.0e-4) * (sR - sM))) {
        usL[ibn] = pl[ibn];
        usL[ibt1] = hll_state(pl[ibt1], pr[ibt1], fl[ibt1], fr[ibt1], sL, sR);
        usL[ibt2] = hll_state(pl[ibt2], pr[ibt2], fl[ibt2], fr[ibt2], sL, sR);
        usR[ibn] = pr[ibn];
        usR[ibt1] = usL[ibt1];
        usR[ibt2] = usL[ibt2];
        sstarL = sM;
        sstarR = sM;
    } else {
        T fac_1 = (pl[irho] * (sL - pl[ivn]) * (sL - sM) - pl[ibn] * pl[ibn]);
        usL[ibn] = pl[ibn];
        usL[ibt1] = dv(pl[ibt1] * (pl[irho] * (sL - pl[ivn]) * (sL - pl[ivn]) - pl[ibn] * pl[ibn]), fac_1);
        usL[ibt2] = dv(pl[ibt2] * (pl[irho] * (sL - pl[ivn]) * (sL - pl[ivn]) - pl[ibn] * pl[ibn]), fac_1);
        fac_1 = (pr[irho] * (sR - pr[ivn]) * (sR - sM) - pr[ibn] * pr[ibn]);
        usR[ibn] = pr[ibn];
        usR[ibt1] = dv(pr[ibt1] * (pr[irho] * (sR - pr[ivn]) * (sR - pr[ivn]) - pr[ibn] * pr[ibn]), fac_1);
        usR[ibt2] = dv(pr[ibt2] * (pr[irho] * (sR - pr[ivn]) * (sR - pr[ivn]) - pr[ibn] * pr[ibn]), fac_1);
    }
    usL[ivn] = usL[irho] * sM;
    usL[ivt1] = usL[ivt1] - dv(usL[ibn] * usL[ibt1] - pl[ibn] * pl[ibt1], sL - sM);
    usL[ivt2] = usL[ivt2] - dv(usL[ibn] * usL[ibt2] - pl[ibn] * pl[ibt2], sL - sM);
    usR[ivn] = usR[irho] * sM;
    usR[ivt1] = usR[ivt1] - dv(usR[ibn] * usR[ibt1] - pr[ibn] * pr[ibt1], sR - sM);
    usR[ivt2] = usR[ivt2] - dv(usR[ibn] * usR[ibt2] - pr[ibn] * pr[ibt2], sR - sM);
    pstL[ivn] = sM;
    pstL[ivt1] = dv(usL[ivt1], usL[irho]);
    pstL[ivt2] = dv(usL[ivt2], usL[irho]);
    pstR[ivn] = sM;
    pstR[ivt1] = dv(usR[ivt1], usR[irho]);
    pstR[ivt2] = dv(usR[ivt2], usR[irho]);
    T pLs = pl[irho] * (sL - pl[ivn]) * (sM - pl[ivn]) + pLt;
    T pRs = pr[irho] * (sR - pr[ivn]) * (sM - pr[ivn]) + pRt;
    T bdotu = pl[ibx] * pl[ivx] + pl[iby] * pl[ivy] + pl[ibz] * pl[ivz];
    T bdotus = usL[ibx] * pstL[ivx] + usL[iby] * pstL[ivy] + usL[ibz] * pstL[ivz];
    usL[itau] = usL[itau] + dv((pLs * sM - pLt * pl[ivn]) - (bdotus - bdotu) * pl[ibn], sL - sM);
    bdotu = pr[ibx] * pr[ivx] + pr[iby] * pr[ivy] + pr[ibz] * pr[ivz];
    bdotus = usR[ibx] * pstR[ivx] + usR[iby] * pstR[ivy] + usR[ibz] * pstR[ivz];
    usR[itau] = usR[itau] + dv((pRs * sM - pRt * pr[ivn]) - (bdotus - bdotu) * pr[ibn], sR - sM);
    if (sstarL >= T(0)) {
#pragma unroll
        for (int i = 1; i <= 8; ++i) fo[i] = fl[i] + sL * (usL[i] - ul[i]);
    } else if (sstarR <= T(0)) {
#pragma unroll
        for (int i = 1; i <= 8; ++i) fo[i] = fr[i] + sR * (usR[i] - ur[i]);
    } else {
        T ussL[9], ussR[9], pssL[9], pssR[9];
        ussL[irho] = usL[irho];
        ussR[irho] = usR[irho];
        const T sqL = dsqrt(usL[irho]), sqR = dsqrt(usR[irho]);
        T fac_1 = T(1) / (sqL + sqR);
        T fac_2 = sign1(pl[ibn]);
        pssL[ivn] = sM;
        pssL[ivt1] = fac_1 * (sqL * pstL[ivt1] + sqR * pstR[ivt1] + (usR[ibt1] - usL[ibt1]) * fac_2);
        pssL[ivt2] = fac_1 * (sqL * pstL[ivt2] + sqR * pstR[ivt2] + (usR[ibt2] - usL[ibt2]) * fac_2);
        const T sqLR = dsqrt(usL[irho] * usR[irho]);
        ussL[ibt1] = fac_1 * (sqL * usR[ibt1] + sqR * usL[ibt1] + sqLR * (pstR[ivt1] - pstL[ivt1]) * fac_2);
        ussL[ibt2] = fac_1 * (sqL * usR[ibt2] + sqR * usL[ibt2] + sqLR * (pstR[ivt2] - pstL[ivt2]) * fac_2);
        ussL[ibn] = usL[ibn];
        ussL[ivn] = ussL[irho] * pssL[ivn];
        ussL[ivt1] = ussL[irho] * pssL[ivt1];
        ussL[ivt2] = ussL[irho] * pssL[ivt2];
        bdotus = usL[ibx] * pstL[ivx] + usL[iby] * pstL[ivy] + usL[ibz] * pstL[ivz];
        T bdotuss = ussL[ibx] * pssL[ivx] + ussL[iby] * pssL[ivy] + ussL[ibz] * pssL[ivz];
        ussL[itau] = usL[itau] - sqL * (bdotus - bdotuss) * fac_2;
        pssR[ivn] = sM;
        pssR[ivt1] = pssL[ivt1];
        pssR[ivt2] = pssL[ivt2];
        ussR[ibt1] = ussL[ibt1];
        ussR[ibt2] = ussL[ibt2];
        ussR[ibn] = usR[ibn];
        ussR[ivn] = ussR[irho] * pssR[ivn];
        ussR[ivt1] = ussR[irho] * pssR[ivt1];
        ussR[ivt2] = ussR[irho] * pssR[ivt2];
        bdotus = usR[ibx] * pstR[ivx] + usR[iby] * pstR[ivy] + usR[ibz] * pstR[ivz];
        bdotuss = ussR[ibx] * pssR[ivx] + ussR[iby] * pssR[ivy] + ussR[ibz] * pssR[ivz];
        ussR[itau] = usR[itau] + sqR * (bdotus - bdotuss) * fac_2;
        if (sM >= T(0)) {
#pragma unroll
            for (int i = 1; i <= 8; ++i) fo[i] = fl[i] + sL * (usL[i] - ul[i]) + sstarL * (ussL[i] - usL[i]);
        } else {
#pragma unroll
            for (int i = 1; i <= 8; ++i) fo[i] = fr[i] + sR * (usR[i] - ur[i]) + sstarR * (ussR[i] - usR[i]);
        }
    }
}

// conserved state of one side, BUILDSTATES spatial.f90:351-362 (same rounding)
template <class T>
__device__ __forceinline__ void cons_state(const T *p, T eps, T *u) {
    T b2 = p[ibx] * p[ibx] + p[iby] * p[iby] + p[ibz] * p[ibz];
    T v2 = p[ivx] * p[ivx] + p[ivy] * p[ivy] + p[ivz] * p[ivz];
    u[irho] = p[irho];
    u[ivx] = p[ivx] * p[irho];
    u[ivy] = p[ivy] * p[irho];
    u[ivz] = p[ivz] * p[irho];
    u[itau] = p[irho] * (T(0.5) * v2 + eps) + T(0.5) * b2;
}

// HLLD of rsolver_module.f90:613-750 with the same arithmetic as hlld_star,
// but the physical fluxes and most conserved components are rebuilt where
// they are used instead of being held across the whole solve (fewer live
// registers, higher occupancy; identical results).
template <class T, int DIR>
__device__ __forceinline__ void hlld_lean(const T *pl, const T *pr, T epsL, T epsR, T *fo, T sL, T sR, T pLt, T pRt) {
    using F = Frame<DIR>;
    constexpr int ivn = F::ivn, ivt1 = F::ivt1, ivt2 = F::ivt2, ibn = F::ibn, ibt1 = F::ibt1, ibt2 = F::ibt2;
    T usL[9], usR[9], pstL[9], pstR[9];
    T sM = sstar_hllc(pLt, pRt, pl[irho], pr[irho], pl[ivn], pr[ivn], sL, sR, pl[ibn], pr[ibn]);
    {
        T ul[9], ur[9];
        cons_state<T>(pl, epsL, ul);
        cons_state<T>(pr, epsR, ur);
#pragma unroll
        for (int i = irho; i <= itau; ++i) usL[i] = dv(ul[i] * (sL - pl[ivn]), sL - sM);
#pragma unroll
        for (int i = irho; i <= itau; ++i) usR[i] = dv(ur[i] * (sR - pr[ivn]), sR - sM);
    }
    T sstarL = sM - dv(dabs(pl[ibn]), dsqrt(usL[irho]));
    T sstarR = sM + dv(dabs(pr[ibn]), dsqrt(usR[irho]));
    if (((sstarL - sL) < T(1.0e-4) * (sM - sL)) || ((sstarR - sR) > -T(1.0e-4) * (sR - sM))) {
        const T flt1 = (pl[ivn] * pl[ibt1] - pl[ivt1] * pl[ibn]), frt1 = (pr[ivn] * pr[ibt1] - pr[ivt1] * pr[ibn]);
        const T flt2 = (pl[ivn] * pl[ibt2] - pl[ivt2] * pl[ibn]), frt2 = (pr[ivn] * pr[ibt2] - pr[ivt2] * pr[ibn]);
        usL[ibn] = pl[ibn];
        usL[ibt1] = hll_state(pl[ibt1], pr[ibt1], flt1, frt1, sL, sR);
        usL[ibt2] = hll_state(pl[ibt2], pr[ibt2], flt2, frt2, sL, sR);
        usR[ibn] = pr[ibn];
        usR[ibt1] = usL[ibt1];
        usR[ibt2] = usL[ibt2];
        sstarL = sM;
        sstarR = sM;
    } else {
        T fac_1 = (pl[irho] * (sL - pl[ivn]) * (sL - sM) - pl[ibn] * pl[ibn]);
        usL[ibn] = pl[ibn];
        usL[ibt1] = dv(pl[ibt1] * (pl[irho] * (sL - pl[ivn]) * (sL - pl[ivn]) - pl[ibn] * pl[ibn]), fac_1);
        usL[ibt2] = dv(pl[ibt2] * (pl[irho] * (sL - pl[ivn]) * (sL - pl[ivn]) - pl[ibn] * pl[ibn]), fac_1);
        fac_1 = (pr[irho] * (sR - pr[ivn]) * (sR - sM) - pr[ibn] * pr[ibn]);
        usR[ibn] = pr[ibn];
        usR[ibt1] = dv(pr[ibt1] * (pr[irho] * (sR - pr[ivn]) * (sR - pr[ivn]) - pr[ibn] * pr[ibn]), fac_1);
        usR[ibt2] = dv(pr[ibt2] * (pr[irho] * (sR - pr[ivn]) * (sR - pr[ivn]) - pr[ibn] * pr[ibn]), fac_1);
    }
    usL[ivn] = usL[irho] * sM;
    usL[ivt1] = usL[ivt1] - dv(usL[ibn] * usL[ibt1] - pl[ibn] * pl[ibt1], sL - sM);
    usL[ivt2] = usL[ivt2] - dv(usL[ibn] * usL[ibt2] - pl[ibn] * pl[ibt2], sL - sM);
    usR[ivn] = usR[irho] * sM;
    usR[ivt1] = usR[ivt1] - dv(usR[ibn] * usR[ibt1] - pr[ibn] * pr[ibt1], sR - sM);
    usR[ivt2] = usR[ivt2] - dv(usR[ibn] * usR[ibt2] - pr[ibn] * pr[ibt2], sR - sM);
    pstL[ivn] = sM;
    pstL[ivt1] = dv(usL[ivt1], usL[irho]);
    pstL[ivt2] = dv(usL[ivt2], usL[irho]);
    pstR[ivn] = sM;
    pstR[ivt1] = dv(usR[ivt1], usR[irho]);
    pstR[ivt2] = dv(usR[ivt2], usR[irho]);
    T pLs = pl[irho] * (sL - pl[ivn]) * (sM - pl[ivn]) + pLt;
    T pRs = pr[irho] * (sR - pr[ivn]) * (sM - pr[ivn]) + pRt;
    T bdotu = pl[ibx] * pl[ivx] + pl[iby] * pl[ivy] + pl[ibz] * pl[ivz];
    T bdotus = usL[ibx] * pstL[ivx] + usL[iby] * pstL[ivy] + usL[ibz] * pstL[ivz];
    usL[itau] = usL[itau] + dv((pLs * sM - pLt * pl[ivn]) - (bdotus - bdotu) * pl[ibn], sL - sM);
    bdotu = pr[ibx] * pr[ivx] + pr[iby] * pr[ivy] + pr[ibz] * pr[ivz];
    bdotus = usR[ibx] * pstR[ivx] + usR[iby] * pstR[ivy] + usR[ibz] * pstR[ivz];
    usR[itau] = usR[itau] + dv((pRs * sM - pRt * pr[ivn]) - (bdotus - bdotu) * pr[ibn], sR - sM);
    // the side whose fan the face lies in; its flux and state are rebuilt here
    const bool left = (sstarL >= T(0)) || !(sstarR <= T(0)) && (sM >= T(0));
    const T *pS = left ? pl : pr;
    const T epsS = left ? epsL : epsR;
    const T s = left ? sL : sR;
    T *usS = left ? usL : usR;
    T uS[9], fS[9];
    build_state<T, DIR>(pS, epsS, uS, fS);
    if (sstarL >= T(0) || sstarR <= T(0)) {
#pragma unroll
        for (int i = 1; i <= 8; ++i) fo[i] = fS[i] + s * (usS[i] - uS[i]);
        return;
    }
    T ussL[9], ussR[9], pssL[9], pssR[9];
    ussL[irho] = usL[irho];
    ussR[irho] = usR[irho];
    const T sqL = dsqrt(usL[irho]), sqR = dsqrt(usR[irho]);
    T fac_1 = T(1) / (sqL + sqR);
    T fac_2 = sign1(pl[ibn]);
    pssL[ivn] = sM;
    pssL[ivt1] = fac_1 * (sqL * pstL[ivt1] + sqR * pstR[ivt1] + (usR[ibt1] - usL[ibt1]) * fac_2);
    pssL[ivt2] = fac_1 * (sqL * pstL[ivt2] + sqR * pstR[ivt2] + (usR[ibt2] - usL[ibt2]) * fac_2);
    const T sqLR = dsqrt(usL[irho] * usR[irho]);
    ussL[ibt1] = fac_1 * (sqL * usR[ibt1] + sqR * usL[ibt1] + sqLR * (pstR[ivt1] - pstL[ivt1]) * fac_2);
    ussL[ibt2] = fac_1 * (sqL * usR[ibt2] + sqR * usL[ibt2] + sqLR * (pstR[ivt2] - pstL[ivt2]) * fac_2);
    ussL[ibn] = usL[ibn];
    ussL[ivn] = ussL[irho] * pssL[ivn];
    ussL[ivt1] = ussL[irho] * pssL[ivt1];
    ussL[ivt2] = ussL[irho] * pssL[ivt2];
    bdotus = usL[ibx] * pstL[ivx] + usL[iby] * pstL[ivy] + usL[ibz] * pstL[ivz];
    T bdotuss = ussL[ibx] * pssL[ivx] + ussL[iby] * pssL[ivy] + ussL[ibz] * pssL[ivz];
    ussL[itau] = usL[itau] - sqL * (bdotus - bdotuss) * fac_2;
    pssR[ivn] = sM;
    pssR[ivt1] = pssL[ivt1];
    pssR[ivt2] = pssL[ivt2];
    ussR[ibt1] = ussL[ibt1];
    ussR[ibt2] = ussL[ibt2];
    ussR[ibn] = usR[ibn];
    ussR[ivn] = ussR[irho] * pssR[ivn];
    ussR[ivt1] = ussR[irho] * pssR[ivt1];
    ussR[ivt2] = ussR[irho] * pssR[ivt2];
    bdotus = usR[ibx] * pstR[ivx] + usR[iby] * pstR[ivy] + usR[ibz] * pstR[ivz];
    bdotuss = ussR[ibx] * pssR[ivx] + ussR[iby] * pssR[ivy] + ussR[ibz] * pssR[ivz];
    ussR[itau] = usR[itau] + sqR * (bdotus - bdotuss) * fac_2;
    const T sst = left ? sstarL : sstarR;
    T *ussS = left ? ussL : ussR;
#pragma unroll
    for (int i = 1; i <= 8; ++i) fo[i] = fS[i] + s * (usS[i] - uS[i]) + sst * (ussS[i] - usS[i]);
}

// One face: BUILDSTATES + the chosen solver (LFNM 133-222, HLLNM 227-326,
// HLLCNM 331-514, HLLDNM 519-767).  pl/pr: primitive L/R states (1-based),
// epsL/R and csL/R from the face EOS.  fo: flux (1-based, 8 comps).
template <class T, int DIR, int RS>
__device__ __forceinline__ void riemann_face(const T *pl, const T *pr, T epsL, T epsR, T csL, T csR, T *fo) {
    using F = Frame<DIR>;
    constexpr int ivn = F::ivn, ibn = F::ibn, ibt1 = F::ibt1, ibt2 = F::ibt2;
    if (RS == RS_HLLD) {
        T cfsL = signalspeed(csL, pl[ibn], pl[ibt1], pl[ibt2], pl[irho]);
        T cfsR = signalspeed(csR, pr[ibn], pr[ibt1], pr[ibt2], pr[irho]);
        T ubar = roe_avg(pl[ivn], pr[ivn], pl[irho], pr[irho]);
        T cbar = roe_avg(cfsL, cfsR, pl[irho], pr[irho]);
        T sL = dmin(pl[ivn] - cfsL, ubar - cbar);
        T sR = dmax(pr[ivn] + cfsR, ubar + cbar);
        if (sL >= T(0) || sR <= T(0)) {
            T u[9];
            build_state<T, DIR>(sL >= T(0) ? pl : pr, sL >= T(0) ? epsL : epsR, u, fo);
            return;
        }
        T b2L = pl[ibx] * pl[ibx] + pl[iby] * pl[iby] + pl[ibz] * pl[ibz];
        T b2R = pr[ibx] * pr[ibx] + pr[iby] * pr[iby] + pr[ibz] * pr[ibz];
        T pLt = pl[itau] + T(0.5) * b2L;
        T pRt = pr[itau] + T(0.5) * b2R;
        hlld_lean<T, DIR>(pl, pr, epsL, epsR, fo, sL, sR, pLt, pRt);
        return;
    }
    T ul[9], ur[9], fl[9], fr[9];
    build_state<T, DIR>(pl, epsL, ul, fl);
    build_state<T, DIR>(pr, epsR, ur, fr);
    T cfsL = signalspeed(csL, pl[ibn], pl[ibt1], pl[ibt2], pl[irho]);
    T cfsR = signalspeed(csR, pr[ibn], pr[ibt1], pr[ibt2], pr[irho]);
    if (RS == RS_LF) {
        T sL = dabs(pl[ivn]) + cfsL, sR = dabs(pr[ivn]) + cfsR;
        T splus = dmax(sL, sR);
#pragma unroll
        for (int i = 1; i <= 8; ++i) fo[i] = T(0.5) * (fl[i] + fr[i] - splus * (ur[i] - ul[i]));
        return;
    }
    T ubar = roe_avg(pl[ivn], pr[ivn], pl[irho], pr[irho]);
    T cbar = roe_avg(cfsL, cfsR, pl[irho], pr[irho]);
    T sL = dmin(pl[ivn] - cfsL, ubar - cbar);
    T sR = dmax(pr[ivn] + cfsR, ubar + cbar);
    if (RS == RS_HLL) {
        if (sL >= T(0)) {
#pragma unroll
            for (int i = 1; i <= 8; ++i) fo[i] = fl[i];
        } else if (sL <= T(0) && sR >= T(0)) {
#pragma unroll
            for (int i = 1; i <= 8; ++i) fo[i] = hll_flux(fl[i], fr[i], ul[i], ur[i], sL, sR);
        } else if (sR <= T(0)) {
#pragma unroll
            for (int i = 1; i <= 8; ++i) fo[i] = fr[i];
        } else {
#pragma unroll
            for (int i = 1; i <= 8; ++i) fo[i] = T(0);
        }
        return;
    }
    if (sL >= T(0)) {
#pragma unroll
        for (int i = 1; i <= 8; ++i) fo[i] = fl[i];
        return;
    }
    if (sR <= T(0)) {
#pragma unroll
        for (int i = 1; i <= 8; ++i) fo[i] = fr[i];
        return;
    }
    T b2L = pl[ibx] * pl[ibx] + pl[iby] * pl[iby] + pl[ibz] * pl[ibz];
    T b2R = pr[ibx] * pr[ibx] + pr[iby] * pr[iby] + pr[ibz] * pr[ibz];
    T pLt = pl[itau] + T(0.5) * b2L;
    T pRt = pr[itau] + T(0.5) * b2R;
    if (RS == RS_HLLC) hllc_star<T, DIR>(pl, pr, ul, ur, fl, fr, fo, sL, sR, pLt, pRt);
    else hlld_star<T, DIR>(pl, pr, ul, ur, fl, fr, fo, sL, sR, pLt, pRt);
}

}  // namespace cumc
