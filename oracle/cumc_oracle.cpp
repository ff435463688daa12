/*
 * cumc_oracle.cpp -- CPU restatement of CUMC3D's per-timestep MHD update.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the B200
 * engine in cumc3d_b200/csrc.  It is built into oracle/_build/liboracle*.so
 * and is loaded only by tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference legs of bench.py.  The product never links or calls it.
 *
 * PARITY UNPINNED: the reference (Fortran 90 + OpenACC, leon-astrophy/cumc3d)
 * cannot be compiled in this environment (no Fortran compiler, no HDF5) and
 * ships no tests, golden vectors or fixtures for this path.  This restatement
 * therefore follows the Fortran routine by routine, loop by loop, in the same
 * floating-point operation order (Fortran left-to-right evaluation, x**2 as
 * x*x), and is checked by invariants instead of reference outputs
 * (tests/test_oracle_invariants.py) and by known answers: the exact
 * ideal-gas Riemann solution on the riemann model's Toro tubes
 * (tests/test_riemann1d.py) and the CP Alfven wave, exact after one period,
 * converging at second order.
 *
 * Layout mirrors the reference: prim(imin:imax,-2:nx+3,-2:ny+3,-2:nz+3) with
 * the variable index fastest.  All arrays start as NaN so that any read of a
 * value the reference leaves undefined shows up in the checked outputs.
 *
 * The scalar type is a template parameter: `double` for parity and timing,
 * `CReal` (a counting double) for exact operation counts per zone-update.
 *
 * Reference files cited below are paths inside leon-astrophy/cumc3d.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdio>
#include <limits>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/cumc3d_gpu.h"

namespace orc {

/* ------------------------------------------------------------------ */
/* scalar types                                                        */
/* ------------------------------------------------------------------ */
struct OpCounts { uint64_t add = 0, mul = 0, div = 0, sqrt = 0, cmp = 0; };
/* counts per phase of the step: 0 the rest, 1 face reconstruction,
 * 2 BUILDSTATES + the Riemann solver, 3 FINDDT */
enum { PH_OTHER = 0, PH_RECON = 1, PH_RIEMANN = 2, PH_DT = 3, N_PHASES = 4 };
static OpCounts g_ops_ph[N_PHASES];
static int g_phase = PH_OTHER;
#define g_ops g_ops_ph[g_phase]
struct PhaseScope {
    int saved;
    explicit PhaseScope(int p) : saved(g_phase) { g_phase = p; }
    ~PhaseScope() { g_phase = saved; }
};

struct CReal {
    double v;
    CReal() : v(0.0) {}
    CReal(double x) : v(x) {}
    explicit operator double() const { return v; }
};
inline CReal operator+(CReal a, CReal b) { g_ops.add++; return CReal(a.v + b.v); }
inline CReal operator-(CReal a, CReal b) { g_ops.add++; return CReal(a.v - b.v); }
inline CReal operator*(CReal a, CReal b) { g_ops.mul++; return CReal(a.v * b.v); }
inline CReal operator/(CReal a, CReal b) { g_ops.div++; return CReal(a.v / b.v); }
inline CReal operator-(CReal a) { return CReal(-a.v); }
inline bool operator<(CReal a, CReal b) { g_ops.cmp++; return a.v < b.v; }
inline bool operator>(CReal a, CReal b) { g_ops.cmp++; return a.v > b.v; }
inline bool operator<=(CReal a, CReal b) { g_ops.cmp++; return a.v <= b.v; }
inline bool operator>=(CReal a, CReal b) { g_ops.cmp++; return a.v >= b.v; }
inline bool operator==(CReal a, CReal b) { g_ops.cmp++; return a.v == b.v; }

inline double dv(double x) { return x; }
inline double dv(CReal x) { return x.v; }

inline double sqrt_(double x) { return std::sqrt(x); }
inline CReal sqrt_(CReal x) { g_ops.sqrt++; return CReal(std::sqrt(x.v)); }
inline double abs_(double x) { return std::fabs(x); }
inline CReal abs_(CReal x) { return CReal(std::fabs(x.v)); }
/* Fortran SIGN(1.0D0, x): magnitude 1 with the sign bit of x */
inline double sign1_(double x) { return std::copysign(1.0, x); }
inline CReal sign1_(CReal x) { return CReal(std::copysign(1.0, x.v)); }
template <class R> inline R min_(R a, R b) { return (b < a) ? b : a; }
template <class R> inline R max_(R a, R b) { return (b > a) ? b : a; }
template <class R> inline R min3_(R a, R b, R c) { return min_(min_(a, b), c); }
template <class R> inline R max3_(R a, R b, R c) { return max_(max_(a, b), c); }

/* variable indices, solver/mhd/setup.f90:39-96 (no custom equations) */
enum { irho = 1, ivx = 2, ivy = 3, ivz = 4, itau = 5, ibx = 6, iby = 7, ibz = 8 };
enum { imin = 1, imax = 8, iex = 9, iey = 10, iez = 11 };
/* face EMF indices, solver/mhd/mhd_module.f90:19-24 */
enum { iyx = 1, izx = 2, ixy = 3, izy = 4, ixz = 5, iyz = 6 };
enum { x_dir = 1, y_dir = 2, z_dir = 3 };

static const double kNaN = std::numeric_limits<double>::quiet_NaN();
static const double small_num = 2.2250738585072014e-308; /* TINY(1.0D0) */

/* SSP-RK3 coefficients, solver/mhd/definition.f90:127-132 */
static const double rk20 = 3.0 / 4.0, rk21 = 1.0 / 4.0, rk22 = 1.0 / 4.0;
static const double rk30 = 1.0 / 3.0, rk31 = 2.0 / 3.0, rk32 = 2.0 / 3.0;

/* WENO-Z constants, solver/mhd/weno_module.f90:16-25 */
static const double smallpara = 1.0e-40;
static const double g_weno_1 = 1.0 / 10.0, g_weno_2 = 6.0 / 10.0, g_weno_3 = 3.0 / 10.0;
static const double r_weno_1 = 13.0 / 12.0, r_weno_2 = 1.0 / 4.0;

/* ------------------------------------------------------------------ */
/* the simulation                                                      */
/* ------------------------------------------------------------------ */
template <class R>
struct Sim {
    cumc_config cfg;
    int nx, ny, nz, n_dim, coord;
    int NX, NY, NZ; /* padded extents n+6 */
    double ggas, cfl;
    std::string err;
    /* cells reconstructed with the positivity fallback (all sweeps, stages) */
    unsigned long long fb_count = 0;

    /* grid (1D), index offset 3 for the -3..n+3 face arrays, 2 for cells */
    std::vector<double> xF_, yF_, zF_;
    std::vector<double> x_, y_, z_, dx_, dy_, dz_, xbar_, dx_cb_, sine_, sinf_, dsine_, dcose_;
    std::vector<double> wx_, wy_, wz_; /* (-2:n+3, 14) */
    int bfac_xin[12], bfac_xout[12], bfac_yin[12], bfac_yout[12], bfac_zin[12], bfac_zout[12];

    /* state */
    std::vector<R> prim, cons, u_old, l_rk, sc, flux;  /* 8 vars */
    std::vector<R> primL, primR, uL, uR, fluxL, fluxR;  /* 8 vars */
    std::vector<R> eps, cs, dpdrho, dpdeps, epsL, epsR, csL, csR;
    std::vector<R> bcell, ecell;  /* 3 vars */
    /* the collapsar model (CUMC_SRC_COLLAPSAR): the self-gravity potential
     * on cells 0..n+1 (natural layout, j fastest), the black hole, and the
     * inner-face mass flux of the x sweep (GETFLUX_X's mflux_x(k,l)) */
    std::vector<double> phi_;
    double m_bh = 0.0, mbh_old = 0.0, r_sh = 0.0, c_code = 1.0;
    bool horizon_hit = false;
    std::vector<R> mflux;
    std::vector<R> eface;         /* 6 vars */
    std::vector<R> efx, efy, efz;

    /* ---- indexing ---- */
    inline size_t c3(int j, int k, int l) const {
        return (size_t)(j + 2) + (size_t)NX * ((size_t)(k + 2) + (size_t)NY * (size_t)(l + 2));
    }
    inline R &P(int i, int j, int k, int l) { return prim[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &U(int i, int j, int k, int l) { return cons[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &UO(int i, int j, int k, int l) { return u_old[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &LR(int i, int j, int k, int l) { return l_rk[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &SC(int i, int j, int k, int l) { return sc[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &FL(int i, int j, int k, int l) { return flux[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &PL(int i, int j, int k, int l) { return primL[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &PR(int i, int j, int k, int l) { return primR[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &UL(int i, int j, int k, int l) { return uL[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &URr(int i, int j, int k, int l) { return uR[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &FXL(int i, int j, int k, int l) { return fluxL[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &FXR(int i, int j, int k, int l) { return fluxR[(size_t)(i - 1) + 8 * c3(j, k, l)]; }
    inline R &E(int j, int k, int l) { return eps[c3(j, k, l)]; }
    inline R &CS(int j, int k, int l) { return cs[c3(j, k, l)]; }
    inline R &BC(int i, int j, int k, int l) { return bcell[(size_t)(i - ibx) + 3 * c3(j, k, l)]; }
    inline R &EC(int i, int j, int k, int l) { return ecell[(size_t)(i - iex) + 3 * c3(j, k, l)]; }
    inline R &EF(int i, int j, int k, int l) { return eface[(size_t)(i - 1) + 6 * c3(j, k, l)]; }
    inline R &EX(int j, int k, int l) { return efx[c3(j, k, l)]; }
    inline R &EY(int j, int k, int l) { return efy[c3(j, k, l)]; }
    inline R &EZ(int j, int k, int l) { return efz[c3(j, k, l)]; }

    double &xF(int j) { return xF_[j + 3]; }
    double &yF(int j) { return yF_[j + 3]; }
    double &zF(int j) { return zF_[j + 3]; }
    double &x(int j) { return x_[j + 2]; }
    double &y(int j) { return y_[j + 2]; }
    double &z(int j) { return z_[j + 2]; }
    double &dx(int j) { return dx_[j + 2]; }
    double &dy(int j) { return dy_[j + 2]; }
    double &dz(int j) { return dz_[j + 2]; }
    double &xbar(int j) { return xbar_[j + 2]; }
    double &dx_cb(int j) { return dx_cb_[j + 2]; }
    double &sine(int j) { return sine_[j + 2]; }
    double &sinf(int j) { return sinf_[j + 3]; }
    double &dsine(int j) { return dsine_[j + 2]; }
    double &dcose(int j) { return dcose_[j + 2]; }
    double *wx(int j) { return &wx_[(size_t)(j + 2) * 14]; }
    double *wy(int j) { return &wy_[(size_t)(j + 2) * 14]; }
    double *wz(int j) { return &wz_[(size_t)(j + 2) * 14]; }

    /* ================================================================ */
    /* setup                                                            */
    /* ================================================================ */
    int init(const cumc_config *c) {
        cfg = *c;
        nx = c->nx; ny = c->ny; nz = c->nz; n_dim = c->n_dim; coord = c->coordinate_flag;
        if (nx < 1 || ny < 1 || nz < 1 || n_dim < 1 || n_dim > 3 || coord < 0 || coord > 2) {
            err = "bad grid extents or flags"; return CUMC_EINVAL;
        }
        if ((n_dim < 2 && ny != 1) || (n_dim < 3 && nz != 1)) { err = "degenerate directions need n=1"; return CUMC_EINVAL; }
        for (int d = 0; d < 3; ++d) {
            int a = c->boundary_flag[2 * d], b = c->boundary_flag[2 * d + 1];
            if ((a == 0) != (b == 0)) { err = "periodic boundary flags must come in pairs"; return CUMC_EINVAL; }
        }
        NX = nx + 6; NY = ny + 6; NZ = nz + 6;
        ggas = c->model.gamma;
        cfl = c->cfl;
        int rc = setup_eqns();
        if (rc) return rc;
        get_grid();
        build_weights();
        size_t n3 = (size_t)NX * NY * NZ;
        auto nanv = [&](std::vector<R> &v, size_t n) { v.assign(n, R(kNaN)); };
        nanv(prim, 8 * n3); nanv(cons, 8 * n3); nanv(u_old, 8 * n3); nanv(l_rk, 8 * n3);
        nanv(sc, 8 * n3); nanv(flux, 8 * n3);
        nanv(primL, 8 * n3); nanv(primR, 8 * n3); nanv(uL, 8 * n3); nanv(uR, 8 * n3);
        nanv(fluxL, 8 * n3); nanv(fluxR, 8 * n3);
        nanv(eps, n3); nanv(cs, n3); nanv(dpdrho, n3); nanv(dpdeps, n3);
        nanv(epsL, n3); nanv(epsR, n3); nanv(csL, n3); nanv(csR, n3);
        nanv(bcell, 3 * n3); nanv(ecell, 3 * n3); nanv(eface, 6 * n3);
        nanv(efx, n3); nanv(efy, n3); nanv(efz, n3);
        return CUMC_OK;
    }

    /* SETUP_EQNS parity factors, solver/mhd/setup.f90:99-325 */
    int setup_eqns() {
        for (int i = 0; i < 12; ++i)
            bfac_xin[i] = bfac_xout[i] = bfac_yin[i] = bfac_yout[i] = bfac_zin[i] = bfac_zout[i] = 1;
        const int *bf = cfg.boundary_flag;
        if (bf[0] == 2) { bfac_xin[ivx] = -1; bfac_xin[ibx] = -1; }
        else if (bf[0] == 3) { bfac_xin[ivx] = -1; bfac_xin[ibx] = -1; bfac_xin[ivz] = -1; bfac_xin[ibz] = -1; }
        else if (bf[0] == 4) { err = "Equatorial symmetry is not allowed for the x-boundary"; return CUMC_EINVAL; }
        if (bf[1] == 2) { bfac_xout[ivx] = -1; bfac_xout[ibx] = -1; }
        else if (bf[1] == 3) { bfac_xout[ivx] = -1; bfac_xout[ibx] = -1; bfac_xout[ivz] = -1; bfac_xout[ibz] = -1; }
        else if (bf[1] == 4) { err = "Equatorial symmetry is not allowed for the x-boundary"; return CUMC_EINVAL; }
        if (bf[2] == 2) { bfac_yin[ivy] = -1; bfac_yin[iby] = -1; }
        else if (bf[2] == 3) { bfac_yin[ivy] = -1; bfac_yin[iby] = -1; bfac_yin[ivz] = -1; bfac_yin[ibz] = -1; }
        else if (bf[2] == 4) { bfac_yin[ivy] = -1; bfac_yin[ibx] = -1; bfac_yin[ibz] = -1; }
        if (bf[3] == 2) { bfac_yout[ivy] = -1; bfac_yout[iby] = -1; }
        else if (bf[3] == 3) { bfac_yout[ivy] = -1; bfac_yout[iby] = -1; bfac_yout[ivz] = -1; bfac_yout[ibz] = -1; }
        else if (bf[3] == 4) { bfac_yout[ivy] = -1; bfac_yout[ibx] = -1; bfac_yout[ibz] = -1; }
        if (bf[4] == 2) { bfac_zin[ivz] = -1; bfac_zin[ibz] = -1; }
        else if (bf[4] == 3) { err = "Axial symmetry is not allowed for the z-boundary"; return CUMC_EINVAL; }
        else if (bf[4] == 4) { bfac_zin[ivz] = -1; bfac_zin[ibx] = -1; bfac_zin[iby] = -1; }
        if (bf[5] == 2) { bfac_zout[ivz] = -1; bfac_zout[ibz] = -1; }
        else if (bf[5] == 3) { err = "Axial symmetry is not allowed for the z-boundary"; return CUMC_EINVAL; }
        else if (bf[5] == 4) { bfac_zout[ivz] = -1; bfac_zout[ibx] = -1; bfac_zout[iby] = -1; }
        int *all[6] = {bfac_xin, bfac_xout, bfac_yin, bfac_yout, bfac_zin, bfac_zout};
        for (int s = 0; s < 6; ++s) {
            int *b = all[s];
            if (b[ivz] * b[iby] * b[ivy] * b[ibz] < 0) { err = "Error in boundary flags for vz and by"; return CUMC_EINVAL; }
            b[iex] = b[ivz] * b[iby];
            if (b[ivx] * b[ibz] * b[ivz] * b[ibx] < 0) { err = "Error in boundary flags for vx and bz"; return CUMC_EINVAL; }
            b[iey] = b[ivx] * b[ibz];
            if (b[ivy] * b[ibx] * b[ivx] * b[iby] < 0) { err = "Error in boundary flags for vy and bx"; return CUMC_EINVAL; }
            b[iez] = b[ivy] * b[ibx];
        }
        return CUMC_OK;
    }

    /* GetGrid, solver/mhd/getgrid.f90:13-98 (face coordinates come from the
     * caller, the CUSTOM_GRID hook; volumes are not used on the stage path) */
    void get_grid() {
        xF_.assign(nx + 7, 0.0); yF_.assign(ny + 7, 0.0); zF_.assign(nz + 7, 0.0);
        for (int j = -3; j <= nx + 3; ++j) xF(j) = cfg.xF[j + 3];
        for (int j = -3; j <= ny + 3; ++j) yF(j) = cfg.yF[j + 3];
        for (int j = -3; j <= nz + 3; ++j) zF(j) = cfg.zF[j + 3];
        x_.assign(NX, kNaN); y_.assign(NY, kNaN); z_.assign(NZ, kNaN);
        dx_.assign(NX, kNaN); dy_.assign(NY, kNaN); dz_.assign(NZ, kNaN);
        xbar_.assign(NX, kNaN); dx_cb_.assign(NX, kNaN);
        sine_.assign(NY, kNaN); sinf_.assign(NY + 1, kNaN); dsine_.assign(NY, kNaN); dcose_.assign(NY, kNaN);
        for (int j = -2; j <= nx + 3; ++j) dx(j) = xF(j) - xF(j - 1);
        for (int j = -2; j <= ny + 3; ++j) dy(j) = yF(j) - yF(j - 1);
        for (int j = -2; j <= nz + 3; ++j) dz(j) = zF(j) - zF(j - 1);
        for (int j = -2; j <= nx + 3; ++j) x(j) = (xF(j) + xF(j - 1)) / 2.0;
        for (int j = -2; j <= ny + 3; ++j) y(j) = (yF(j) + yF(j - 1)) / 2.0;
        for (int j = -2; j <= nz + 3; ++j) z(j) = (zF(j) + zF(j - 1)) / 2.0;
        for (int j = -1; j <= nx + 3; ++j) {
            dx_cb(j) = xF(j) * xF(j) * xF(j) - xF(j - 1) * xF(j - 1) * xF(j - 1);
            xbar(j) = (dx_cb(j) / 3.0) / (x(j) * dx(j));
        }
        for (int k = -1; k <= ny + 3; ++k) {
            dcose(k) = -(std::cos(yF(k)) - std::cos(yF(k - 1)));
            dsine(k) = (std::sin(yF(k)) - std::sin(yF(k - 1)));
        }
        for (int k = -2; k <= ny + 3; ++k) sine(k) = std::sin(y(k));
        for (int k = -3; k <= ny + 3; ++k) sinf(k) = std::sin(yF(k));
        if (cfg.fixpole && coord == 2) {
            yF(0) = 0.0; yF(ny) = 4.0 * std::atan(1.0);
            sinf(0) = 0.0; sinf(ny) = 0.0;
        }
    }

    /* TVD_WEIGHT tvd_module.f90:25-55; PPM_WEIGHT/PPM_INTERPOLANT
     * ppmc_module.f90:17-145; WENO_WEIGHT/WENO_INTERPOLANT weno_module.f90:35-149 */
    static void ppm_interpolant(double dm2, double dm1, double dc, double dp1, double dp2, double *w) {
        double a1R = dc / (dc + dp1);
        double a1L = dm1 / (dm1 + dc);
        double aR = 2.0 * dp1 * dc / (dp1 + dc);
        double aL = 2.0 * dc * dm1 / (dc + dm1);
        double deltaXR = dm1 + dc + dp1 + dp2;
        double deltaXL = dm2 + dm1 + dc + dp1;
        double z1R = (dm1 + dc) / (2.0 * dc + dp1);
        double z1L = (dm2 + dm1) / (2.0 * dm1 + dc);
        double zR = (dp2 + dp1) / (2.0 * dp1 + dc);
        double zL = (dp1 + dc) / (2.0 * dc + dm1);
        double cc1 = dc / (dm1 + dc + dp1);
        double cp1 = dp1 / (dc + dp1 + dp2);
        double cm1 = dm1 / (dm2 + dm1 + dc);
        double cc2 = (2.0 * dm1 + dc) / (dp1 + dc);
        double cp2 = (2.0 * dc + dp1) / (dp2 + dp1);
        double cm2 = (2.0 * dm2 + dm1) / (dc + dm1);
        double cc3 = (dc + 2.0 * dp1) / (dm1 + dc);
        double cp3 = (dp1 + 2.0 * dp2) / (dc + dp1);
        double cm3 = (dm1 + 2.0 * dc) / (dm2 + dm1);
        w[0] = a1L;
        w[1] = aL * (z1L - zL) / deltaXL;
        w[2] = (-dm1 * z1L) / deltaXL;
        w[3] = dc * zL / deltaXL;
        w[4] = a1R;
        w[5] = aR * (z1R - zR) / deltaXR;
        w[6] = (-dc * z1R) / deltaXR;
        w[7] = dp1 * zR / deltaXR;
        w[8] = cm1 * cm2;
        w[9] = cm1 * cm3;
        w[10] = cc1 * cc2;
        w[11] = cc1 * cc3;
        w[12] = cp1 * cp2;
        w[13] = cp1 * cp3;
    }
    static void weno_interpolant(double dm2, double dm1, double dc, double dp1, double dp2, double *w) {
        double alpha12 = dp2 / (dp1 + dp2);
        double alpha01 = dp1 / (dc + dp1);
        double alpha10 = dc / (dm1 + dc);
        double alpha21 = dm1 / (dm2 + dm1);
        w[0] = (1.0 - alpha01);
        w[1] = alpha01;
        w[2] = (1.0 - alpha12);
        w[3] = alpha12;
        w[4] = (1.0 - alpha10);
        w[5] = alpha10;
        w[6] = (1.0 - alpha21);
        w[7] = alpha21;
        w[8] = (1.0 - alpha21);
        w[9] = alpha12;
    }
    void build_weights() {
        wx_.assign((size_t)NX * 14, kNaN); wy_.assign((size_t)NY * 14, kNaN); wz_.assign((size_t)NZ * 14, kNaN);
        int rc = cfg.recon;
        auto fill = [&](int n, double *(Sim::*w)(int), double &(Sim::*d)(int)) {
            if (rc == CUMC_RECON_WENO || rc == CUMC_RECON_PPM) {
                for (int j = 0; j <= n + 1; ++j) {
                    double dm2 = (this->*d)(j - 2), dm1 = (this->*d)(j - 1), dc = (this->*d)(j),
                           dp1 = (this->*d)(j + 1), dp2 = (this->*d)(j + 2);
                    if (rc == CUMC_RECON_WENO) weno_interpolant(dm2, dm1, dc, dp1, dp2, (this->*w)(j));
                    else ppm_interpolant(dm2, dm1, dc, dp1, dp2, (this->*w)(j));
                }
            } else {
                for (int j = -1; j <= n + 2; ++j) {
                    (this->*w)(j)[0] = ((this->*d)(j) + (this->*d)(j + 1)) / (this->*d)(j);
                    (this->*w)(j)[1] = ((this->*d)(j) + (this->*d)(j - 1)) / (this->*d)(j);
                }
            }
        };
        fill(nx, &Sim::wx, &Sim::dx);
        fill(ny, &Sim::wy, &Sim::dy);
        fill(nz, &Sim::wz, &Sim::dz);
    }

    /* ================================================================ */
    /* model hooks                                                      */
    /* ================================================================ */
    /* EOSEPSILON_NM model/riemann/src/getepsilon.f90:4-16 */
    inline R eos_eps(R rho, R p) { return p / rho / (ggas - 1.0); }
    /* EOSSOUNDSPEED model/riemann/src/soundspeed.f90:4-21 */
    inline R eos_cs(R p, R rho, R e) {
        R dpdden = e * (ggas - 1.0);
        R dpdint = rho * (ggas - 1.0);
        return sqrt_(dpdden + dpdint * p / (rho * rho));
    }

    /* CUSTOM_CHECKRHO */
    void custom_checkrho() {
        const cumc_model &m = cfg.model;
        if (m.floor_kind == CUMC_FLOOR_EPS) {
            /* model/riemann/src/custom.f90:103-127 */
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j) E(j, k, l) = max_(E(j, k, l), R(0.0));
        } else if (m.floor_kind == CUMC_FLOOR_TORUS) {
            /* model/torus-cyn/src/custom.f90:240-275, uniform floor arrays */
            const double rho_floor = m.rho_floor, eps_floor = m.eps_floor;
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j) {
                        R diff = P(irho, j, k, l) - rho_floor;
                        R factor = max_(sign1_(diff), R(0.0));
                        P(irho, j, k, l) = factor * P(irho, j, k, l) + (1.0 - factor) * rho_floor;
                        for (int i = ivx; i <= ivz; ++i) P(i, j, k, l) = factor * P(i, j, k, l);
                        E(j, k, l) = factor * E(j, k, l) + (1.0 - factor) * eps_floor;
                        if (E(j, k, l) < 0.0) E(j, k, l) = eps_floor;
                    }
        } else if (m.floor_kind == CUMC_FLOOR_COLLAPSAR) {
            /* model/collapsar/src/custom.f90:289-304: prim(irho:ivz) blended
             * with the atmosphere prim_a = (rho_a, 0, 0, 0), eps with eps_a */
            const double rho_a = m.rho_floor, eps_a = m.eps_floor;
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j) {
                        R diff = P(irho, j, k, l) - rho_a;
                        R factor = max_(sign1_(diff), R(0.0));
                        P(irho, j, k, l) = factor * P(irho, j, k, l) + (1.0 - factor) * rho_a;
                        for (int i = ivx; i <= ivz; ++i) P(i, j, k, l) = factor * P(i, j, k, l) + (1.0 - factor) * 0.0;
                        E(j, k, l) = factor * E(j, k, l) + (1.0 - factor) * eps_a;
                        if (E(j, k, l) < 0.0) E(j, k, l) = eps_a;
                    }
        }
    }

    /* FINDPRESSURE: model/riemann/src/findpressure.f90:7-51 and
     * model/torus-cyn/src/findpressure.f90:7-37 (the floor branch) */
    void findpressure() {
        const cumc_model &m = cfg.model;
        const bool torus = (m.floor_kind == CUMC_FLOOR_TORUS);
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = -2; l <= nz + 3; ++l)
            for (int k = -2; k <= ny + 3; ++k)
                for (int j = -2; j <= nx + 3; ++j) {
                    size_t c = c3(j, k, l);
                    if (!torus || P(irho, j, k, l) > m.rho_floor) {
                        P(itau, j, k, l) = P(irho, j, k, l) * eps[c] * (ggas - 1.0);
                        dpdrho[c] = eps[c] * (ggas - 1.0);
                        dpdeps[c] = P(irho, j, k, l) * (ggas - 1.0);
                    } else {
                        P(itau, j, k, l) = R(m.p_floor);
                        dpdrho[c] = R(m.eps_floor * (ggas - 1.0));
                        dpdeps[c] = R(m.rho_floor * (ggas - 1.0));
                    }
                    cs[c] = sqrt_(dpdrho[c] + dpdeps[c] * P(itau, j, k, l) / (P(irho, j, k, l) * P(irho, j, k, l)));
                }
    }

    /* CUSTOM_SOURCE */
    void custom_source() {
        const cumc_model &m = cfg.model;
        if (m.source_kind == CUMC_SRC_CONST_GY) {
            /* model/riemann/src/custom.f90:143-155 */
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j)
                        SC(ivy, j, k, l) = SC(ivy, j, k, l) - m.g_const * P(irho, j, k, l);
        } else if (m.source_kind == CUMC_SRC_PM_CYL) {
            /* model/torus-cyn/src/custom.f90:298-314 */
            const double r_sh = m.r_sh;
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j) {
                        R diff = P(irho, j, k, l) - m.rho_floor;
                        R factor = max_(sign1_(diff), R(0.0));
                        R radius = sqrt_(R(x(j) * x(j) + z(l) * z(l)));
                        R dphidr = R(x(j)) / radius / ((radius - r_sh) * (radius - r_sh));
                        R dphidz = R(z(l)) / radius / ((radius - r_sh) * (radius - r_sh));
                        SC(ivx, j, k, l) = SC(ivx, j, k, l) + (-(factor * P(irho, j, k, l) * dphidr));
                        SC(ivz, j, k, l) = SC(ivz, j, k, l) + (-(factor * P(irho, j, k, l) * dphidz));
                        SC(itau, j, k, l) = SC(itau, j, k, l) +
                            (-(factor * P(irho, j, k, l) * (P(ivx, j, k, l) * dphidr + P(ivz, j, k, l) * dphidz)));
                    }
        } else if (m.source_kind == CUMC_SRC_COLLAPSAR) {
            /* model/collapsar/src/custom.f90:355-385: the potential's gradient
             * (first_derivative, custom.f90:402-409) plus the black hole */
            const long long px = nx + 2, py = (long long)(nx + 2) * (ny + 2);
            auto ph = [&](int j, int k, int l) { return R(phi_[j + px * k + py * l]); };
            auto fd = [](R xm1, R xc, R xp1, R fm1, R fc, R fp1) {
                R h2 = xp1 - xc, h1 = xc - xm1;
                return ((fp1 - fc) * h1 * h1 + (fc - fm1) * h2 * h2) / (h1 * h2 * (h1 + h2));
            };
            const double mb = m_bh, rs = r_sh;
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j) {
                        R diff = P(irho, j, k, l) - m.rho_floor;
                        R factor = max_(sign1_(diff), R(0.0));
                        R dphidx = fd(R(x(j - 1)), R(x(j)), R(x(j + 1)), ph(j - 1, k, l), ph(j, k, l), ph(j + 1, k, l));
                        R dphidy = fd(R(y(k - 1)), R(y(k)), R(y(k + 1)), ph(j, k - 1, l), ph(j, k, l), ph(j, k + 1, l));
                        R dphidz = fd(R(z(l - 1)), R(z(l)), R(z(l + 1)), ph(j, k, l - 1), ph(j, k, l), ph(j, k, l + 1));
                        dphidx = dphidx + mb / ((x(j) - rs) * (x(j) - rs));
                        const R rho = P(irho, j, k, l);
                        SC(ivx, j, k, l) = SC(ivx, j, k, l) - factor * rho * dphidx;
                        SC(ivy, j, k, l) = SC(ivy, j, k, l) - factor * rho * dphidy / x(j);
                        SC(ivz, j, k, l) = SC(ivz, j, k, l) - factor * rho * dphidz / x(j) / sine(k);
                        SC(itau, j, k, l) = SC(itau, j, k, l) -
                            factor * rho * (P(ivx, j, k, l) * dphidx + P(ivy, j, k, l) * dphidy / x(j) +
                                            P(ivz, j, k, l) * dphidz / x(j) / sine(k));
                    }
        } else if (m.source_kind == CUMC_SRC_PM_SPH) {
            /* model/torus-sph/src/custom.f90 CUSTOM_SOURCE (radial form) */
            const double r_sh = m.r_sh;
#pragma omp parallel for collapse(2) schedule(static)
            for (int l = 1; l <= nz; ++l)
                for (int k = 1; k <= ny; ++k)
                    for (int j = 1; j <= nx; ++j) {
                        R diff = P(irho, j, k, l) - m.rho_floor;
                        R factor = max_(sign1_(diff), R(0.0));
                        R dphidr = R(1.0) / R((x(j) - r_sh) * (x(j) - r_sh));
                        SC(ivx, j, k, l) = SC(ivx, j, k, l) + (-(factor * P(irho, j, k, l) * dphidr));
                        SC(itau, j, k, l) = SC(itau, j, k, l) + (-(factor * P(irho, j, k, l) * P(ivx, j, k, l) * dphidr));
                    }
        }
    }

    /* CUSTOM_BOUNDARY_X/Y/Z */
    void custom_boundary() {
        const int kind = cfg.model.bc_kind;
        if (kind == CUMC_BC_TORUS_CYL || kind == CUMC_BC_TORUS_SPH) {
            /* model/torus-cyn/src/custom.f90:146-170 */
            for (int l = -2; l <= nz + 3; ++l)
                for (int k = -2; k <= ny + 3; ++k)
                    for (int j = 1; j <= 3; ++j) {
                        P(ivx, 1 - j, k, l) = min_(P(ivx, 1 - j, k, l), R(0.0));
                        P(ivx, nx + j, k, l) = max_(P(ivx, nx + j, k, l), R(0.0));
                    }
        }
        if (kind == CUMC_BC_TORUS_CYL) {
            /* model/torus-cyn/src/custom.f90:184-208 */
            for (int l = 1; l <= 3; ++l)
                for (int k = -2; k <= ny + 3; ++k)
                    for (int j = -2; j <= nx + 3; ++j) {
                        P(ivz, j, k, 1 - l) = min_(P(ivz, j, k, 1 - l), R(0.0));
                        P(ivz, j, k, nz + l) = max_(P(ivz, j, k, nz + l), R(0.0));
                    }
        }
    }

    /* ================================================================ */
    /* conversions, solver/mhd/fromrvetou.f90                           */
    /* ================================================================ */
    template <class F>
    void face_to_cell_b(F &&face) {
        /* fromrvetou.f90:48-90 (from prim) and 153-195 (from cons) */
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    if (coord == 0) {
                        BC(ibx, j, k, l) = 0.5 * (face(ibx, j, k, l) + face(ibx, j - 1, k, l));
                        BC(iby, j, k, l) = 0.5 * (face(iby, j, k, l) + face(iby, j, k - 1, l));
                        BC(ibz, j, k, l) = 0.5 * (face(ibz, j, k, l) + face(ibz, j, k, l - 1));
                    } else if (coord == 1) {
                        BC(ibx, j, k, l) = (xF(j) * face(ibx, j, k, l) + xF(j - 1) * face(ibx, j - 1, k, l)) / (xF(j) + xF(j - 1));
                        BC(iby, j, k, l) = 0.5 * (face(iby, j, k, l) + face(iby, j, k - 1, l));
                        BC(ibz, j, k, l) = 0.5 * (face(ibz, j, k, l) + face(ibz, j, k, l - 1));
                    } else {
                        BC(ibx, j, k, l) = 1.5 * dx(j) / dx_cb(j) *
                            ((xF(j) * xF(j)) * face(ibx, j, k, l) + (xF(j - 1) * xF(j - 1)) * face(ibx, j - 1, k, l));
                        BC(iby, j, k, l) = 0.5 * dy(k) / dcose(k) *
                            (sinf(k) * face(iby, j, k, l) + sinf(k - 1) * face(iby, j, k - 1, l));
                        BC(ibz, j, k, l) = 0.5 * (face(ibz, j, k, l) + face(ibz, j, k, l - 1));
                    }
                }
    }

    /* FROMRVETOU fromrvetou.f90:21-121 */
    void fromrvetou() {
        face_to_cell_b([&](int i, int j, int k, int l) -> R { return P(i, j, k, l); });
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    R vsquare = P(ivx, j, k, l) * P(ivx, j, k, l) + P(ivy, j, k, l) * P(ivy, j, k, l) + P(ivz, j, k, l) * P(ivz, j, k, l);
                    R bsquare = BC(ibx, j, k, l) * BC(ibx, j, k, l) + BC(iby, j, k, l) * BC(iby, j, k, l) + BC(ibz, j, k, l) * BC(ibz, j, k, l);
                    U(irho, j, k, l) = P(irho, j, k, l);
                    for (int i = ivx; i <= ivz; ++i) U(i, j, k, l) = P(i, j, k, l) * P(irho, j, k, l);
                    U(itau, j, k, l) = P(irho, j, k, l) * (E(j, k, l) + 0.5 * vsquare) + 0.5 * bsquare;
                    for (int i = ibx; i <= ibz; ++i) U(i, j, k, l) = P(i, j, k, l);
                }
    }

    /* FROMUTORVE fromrvetou.f90:126-227 */
    void fromutorve() {
        face_to_cell_b([&](int i, int j, int k, int l) -> R { return U(i, j, k, l); });
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    P(irho, j, k, l) = U(irho, j, k, l);
                    for (int i = ivx; i <= ivz; ++i) P(i, j, k, l) = U(i, j, k, l) / U(irho, j, k, l);
                    for (int i = ibx; i <= ibz; ++i) P(i, j, k, l) = U(i, j, k, l);
                    R bsquare = BC(ibx, j, k, l) * BC(ibx, j, k, l) + BC(iby, j, k, l) * BC(iby, j, k, l) + BC(ibz, j, k, l) * BC(ibz, j, k, l);
                    R vsquare = P(ivx, j, k, l) * P(ivx, j, k, l) + P(ivy, j, k, l) * P(ivy, j, k, l) + P(ivz, j, k, l) * P(ivz, j, k, l);
                    E(j, k, l) = (U(itau, j, k, l) - 0.5 * bsquare) / U(irho, j, k, l) - 0.5 * vsquare;
                }
    }

    /* ================================================================ */
    /* ghost fill, solver/mhd/boundary.f90                              */
    /* ================================================================ */
    /* One array (or one component list) filled x then y then z exactly as
     * BOUNDARYP_NM (397-770) and BOUNDARY1D_NM (29-389) do. */
    template <class A>
    void fill_x(A &&a, int sin_, int sout_) {
        const int *bf = cfg.boundary_flag;
        for (int l = -2; l <= nz + 3; ++l)
            for (int k = -2; k <= ny + 3; ++k)
                for (int j = 1; j <= 3; ++j) {
                    if (bf[0] == 0) a(1 - j, k, l) = R(a(nx + 1 - j, k, l));
                    else if (bf[0] == 1) a(1 - j, k, l) = R(a(1, k, l));
                    else a(1 - j, k, l) = R(double(sin_)) * a(j, k, l);
                }
        for (int l = -2; l <= nz + 3; ++l)
            for (int k = -2; k <= ny + 3; ++k)
                for (int j = 1; j <= 3; ++j) {
                    if (bf[1] == 0) a(nx + j, k, l) = R(a(j, k, l));
                    else if (bf[1] == 1) a(nx + j, k, l) = R(a(nx, k, l));
                    else a(nx + j, k, l) = R(double(sout_)) * a(nx + 1 - j, k, l);
                }
    }
    /* y_out_flag lets BOUNDARY1D_NM reproduce its y-outer test of
     * boundary_flag(3) for the periodic case (boundary.f90:243) */
    template <class A>
    void fill_y(A &&a, int sin_, int sout_, bool eps_quirk) {
        const int *bf = cfg.boundary_flag;
        for (int l = -2; l <= nz + 3; ++l)
            for (int k = 1; k <= 3; ++k)
                for (int j = -2; j <= nx + 3; ++j) {
                    if (bf[2] == 0) a(j, 1 - k, l) = R(a(j, ny + 1 - k, l));
                    else if (bf[2] == 1) a(j, 1 - k, l) = R(a(j, 1, l));
                    else a(j, 1 - k, l) = R(double(sin_)) * a(j, k, l);
                }
        int mode = eps_quirk ? (bf[2] == 0 ? 0 : (bf[3] == 1 ? 1 : (bf[3] >= 2 ? 2 : -1))) : bf[3];
        for (int l = -2; l <= nz + 3; ++l)
            for (int k = 1; k <= 3; ++k)
                for (int j = -2; j <= nx + 3; ++j) {
                    if (mode == 0) a(j, ny + k, l) = R(a(j, k, l));
                    else if (mode == 1) a(j, ny + k, l) = R(a(j, ny, l));
                    else if (mode >= 2) a(j, ny + k, l) = R(double(sout_)) * a(j, ny + 1 - k, l);
                }
    }
    template <class A>
    void fill_z(A &&a, int sin_, int sout_) {
        const int *bf = cfg.boundary_flag;
        for (int l = 1; l <= 3; ++l)
            for (int k = -2; k <= ny + 3; ++k)
                for (int j = -2; j <= nx + 3; ++j) {
                    if (bf[4] == 0) a(j, k, 1 - l) = R(a(j, k, nz + 1 - l));
                    else if (bf[4] == 1) a(j, k, 1 - l) = R(a(j, k, 1));
                    else a(j, k, 1 - l) = R(double(sin_)) * a(j, k, l);
                }
        for (int l = 1; l <= 3; ++l)
            for (int k = -2; k <= ny + 3; ++k)
                for (int j = -2; j <= nx + 3; ++j) {
                    if (bf[5] == 0) a(j, k, nz + l) = R(a(j, k, l));
                    else if (bf[5] == 1) a(j, k, nz + l) = R(a(j, k, nz));
                    else a(j, k, nz + l) = R(double(sout_)) * a(j, k, nz + 1 - l);
                }
    }

    /* BOUNDARYP_NM boundary.f90:397-770 + custom hooks, then
     * BOUNDARY1D_NM(epsilon, even...) boundary.f90:5-13 */
    void boundary() {
        auto pv = [&](int i) { return [this, i](int j, int k, int l) -> R & { return P(i, j, k, l); }; };
        auto bv = [&](int i) { return [this, i](int j, int k, int l) -> R & { return BC(i, j, k, l); }; };
        /* x pass: hydro 1..5, bcell, prim(iby), prim(ibz) */
        for (int i = imin; i <= itau; ++i) fill_x(pv(i), bfac_xin[i], bfac_xout[i]);
        for (int i = ibx; i <= ibz; ++i) fill_x(bv(i), bfac_xin[i], bfac_xout[i]);
        fill_x(pv(iby), bfac_xin[iby], bfac_xout[iby]);
        fill_x(pv(ibz), bfac_xin[ibz], bfac_xout[ibz]);
        /* option: a periodic direction also carries its normal face field, so
         * face 0 is face n (the reference leaves face 0 at its initial value) */
        const int *bf = cfg.boundary_flag;
        const bool fixn = cfg.fix_periodic_normal_faces != 0;
        if (fixn && bf[0] == 0) fill_x(pv(ibx), 1, 1);
        /* y pass: hydro, bcell, prim(ibx), prim(ibz) */
        for (int i = imin; i <= itau; ++i) fill_y(pv(i), bfac_yin[i], bfac_yout[i], false);
        for (int i = ibx; i <= ibz; ++i) fill_y(bv(i), bfac_yin[i], bfac_yout[i], false);
        fill_y(pv(ibx), bfac_yin[ibx], bfac_yout[ibx], false);
        fill_y(pv(ibz), bfac_yin[ibz], bfac_yout[ibz], false);
        if (fixn && bf[2] == 0) fill_y(pv(iby), 1, 1, false);
        /* z pass: hydro, bcell, prim(ibx), prim(iby) */
        for (int i = imin; i <= itau; ++i) fill_z(pv(i), bfac_zin[i], bfac_zout[i]);
        for (int i = ibx; i <= ibz; ++i) fill_z(bv(i), bfac_zin[i], bfac_zout[i]);
        fill_z(pv(ibx), bfac_zin[ibx], bfac_zout[ibx]);
        fill_z(pv(iby), bfac_zin[iby], bfac_zout[iby]);
        if (fixn && bf[4] == 0) fill_z(pv(ibz), 1, 1);
        custom_boundary();
        /* epsilon: all-even parity */
        auto ev = [this](int j, int k, int l) -> R & { return E(j, k, l); };
        fill_x(ev, 1, 1);
        fill_y(ev, 1, 1, true);
        fill_z(ev, 1, 1);
    }

    /* UPDATE update.f90:12-33: FINDPRESSURE (+ empty CUSTOM_UPDATE) */
    void update() { findpressure(); }

    /* ================================================================ */
    /* reconstruction                                                   */
    /* ================================================================ */
    /* PPMC ppmc_module.f90:359-464 */
    static void ppmc(const double *wgt, R vm2, R vm1, R vc, R vp1, R vp2, R &vm_out, R &vp_out) {
        const double a0m = wgt[0], a1m = wgt[1], a2m = wgt[2], a3m = wgt[3];
        const double a0p = wgt[4], a1p = wgt[5], a2p = wgt[6], a3p = wgt[7];
        const double b0m = wgt[8], b1m = wgt[9], b0c = wgt[10], b1c = wgt[11], b0p = wgt[12], b1p = wgt[13];
        R deltap1 = b0p * (vp2 - vp1) + b1p * (vp1 - vc);
        R deltac = b0c * (vp1 - vc) + b1c * (vc - vm1);
        R deltam1 = b0m * (vc - vm1) + b1m * (vm1 - vm2);
        R dmc, dmp1, dmm1, condition;
        condition = (vp1 - vc) * (vc - vm1);
        if (condition > 0.0) dmc = min3_(abs_(deltac), 2.0 * abs_(vc - vm1), 2.0 * abs_(vc - vp1)) * sign1_(deltac);
        else dmc = R(0.0);
        condition = (vp2 - vp1) * (vp1 - vc);
        if (condition > 0.0) dmp1 = min3_(abs_(deltap1), 2.0 * abs_(vp1 - vc), 2.0 * abs_(vp1 - vp2)) * sign1_(deltap1);
        else dmp1 = R(0.0);
        condition = (vc - vm1) * (vm1 - vm2);
        if (condition > 0.0) dmm1 = min3_(abs_(deltam1), 2.0 * abs_(vm1 - vm2), 2.0 * abs_(vm1 - vc)) * sign1_(deltam1);
        else dmm1 = R(0.0);
        vp_out = vc + a0p * (vp1 - vc) + a1p * (vp1 - vc) + a2p * dmp1 + a3p * dmc;
        vm_out = vm1 + a0m * (vc - vm1) + a1m * (vc - vm1) + a2m * dmc + a3m * dmm1;
        R vl = vm_out, vr = vp_out;
        if ((vr - vc) * (vc - vl) <= 0.0) {
            vp_out = vc;
            vm_out = vc;
        } else {
            condition = (vr - vl) * (vl - 3.0 * vc + 2.0 * vr);
            if (condition < 0.0) vm_out = 3.0 * vc - 2.0 * vr;
            condition = (vp_out - vm_out) * (3.0 * vc - 2.0 * vl - vr);
            if (condition < 0.0) vp_out = 3.0 * vc - 2.0 * vl;
        }
    }

    /* WENO (WENO-Z) weno_module.f90:315-408 */
    static void weno(const double *wgt, R vm2, R vm1, R vc, R vp1, R vp2, R &vm_out, R &vp_out) {
        R U01 = wgt[0] * vc + wgt[1] * vp1;
        R U12 = wgt[2] * vp1 + wgt[3] * vp2;
        R U10 = wgt[4] * vm1 + wgt[5] * vc;
        R U21 = wgt[6] * vm2 + wgt[7] * vm1;
        R U00 = vm1 + wgt[8] * (vm1 - vm2);
        R U11 = vp1 + wgt[9] * (vp1 - vp2);
        R P1 = (6.0 * vc - 1.0 * U10 - 2.0 * U00) / 3.0;
        R P2 = (-1.0 * U10 + 2.0 * vc + 2.0 * U01) / 3.0;
        R P3 = (2.0 * U01 + 2.0 * vp1 - 1.0 * U12) / 3.0;
        R t1 = 2.0 * U10 - 2.0 * U00, t2 = 4.0 * vc - 2.0 * U10 - 2.0 * U00;
        R B1 = r_weno_1 * (t1 * t1) + r_weno_2 * (t2 * t2);
        R t3 = 2.0 * U10 - 4.0 * vc + 2.0 * U01, t4 = -2.0 * U10 + 2.0 * U01;
        R B2 = r_weno_1 * (t3 * t3) + r_weno_2 * (t4 * t4);
        R t5 = 2.0 * U01 - 4.0 * vp1 + 2.0 * U12, t6 = -6.0 * U01 + 8.0 * vp1 - 2.0 * U12;
        R B3 = r_weno_1 * (t5 * t5) + r_weno_2 * (t6 * t6);
        R tau5 = abs_(B1 - B3);
        R q1 = tau5 / (smallpara + B1), q2 = tau5 / (smallpara + B2), q3 = tau5 / (smallpara + B3);
        R w1 = g_weno_1 * (1.0 + q1 * q1);
        R w2 = g_weno_2 * (1.0 + q2 * q2);
        R w3 = g_weno_3 * (1.0 + q3 * q3);
        vp_out = (w1 * P1 + w2 * P2 + w3 * P3) / (w1 + w2 + w3);
        P1 = (6.0 * vc - 1.0 * U01 - 2.0 * U11) / 3.0;
        P2 = (-1.0 * U01 + 2.0 * vc + 2.0 * U10) / 3.0;
        P3 = (2.0 * U10 + 2.0 * vm1 - 1.0 * U21) / 3.0;
        t1 = 2.0 * U01 - 2.0 * U11; t2 = 4.0 * vc - 2.0 * U01 - 2.0 * U11;
        B1 = r_weno_1 * (t1 * t1) + r_weno_2 * (t2 * t2);
        t3 = 2.0 * U01 - 4.0 * vc + 2.0 * U10; t4 = 2.0 * U01 - 2.0 * U10;
        B2 = r_weno_1 * (t3 * t3) + r_weno_2 * (t4 * t4);
        t5 = 2.0 * U10 - 4.0 * vm1 + 2.0 * U21; t6 = 8.0 * vm1 - 6.0 * U10 - 2.0 * U21;
        B3 = r_weno_1 * (t5 * t5) + r_weno_2 * (t6 * t6);
        tau5 = abs_(B1 - B3);
        q1 = tau5 / (smallpara + B1); q2 = tau5 / (smallpara + B2); q3 = tau5 / (smallpara + B3);
        w1 = g_weno_1 * (1.0 + q1 * q1);
        w2 = g_weno_2 * (1.0 + q2 * q2);
        w3 = g_weno_3 * (1.0 + q3 * q3);
        vm_out = (w1 * P1 + w2 * P2 + w3 * P3) / (w1 + w2 + w3);
    }

    /* TVD tvd_module.f90:279-344 */
    static void tvd(int lim, const double *wgt, R vm, R vc, R vp, R &vm_out, R &vp_out) {
        const double cf = wgt[0], cb = wgt[1];
        R dqf = 2.0 * (vp - vc) / cf;
        R dqb = 2.0 * (vc - vm) / cb;
        R slope;
        if (lim == CUMC_RECON_TVD_MM) {
            slope = 0.5 * (sign1_(dqf) + sign1_(dqb)) * min_(abs_(dqf), abs_(dqb));
        } else if (lim == CUMC_RECON_TVD_VL) {
            R dq2 = dqf * dqb;
            if (dq2 <= 0.0) slope = R(0.0);
            else slope = (dq2 * (cf * dqb + cb * dqf) / (dqb * dqb + dqf * dqf + dq2 * (cf + cb - 2.0)));
        } else {
            if (dqf == 0.0) slope = R(0.0);
            else {
                R v_tvd = dqb / dqf;
                slope = max_(R(0.0), min3_(0.5 * (1.0 + v_tvd), R(cf), cb * v_tvd));
                slope = dqf * slope;
            }
        }
        vp_out = vc + 0.5 * slope;
        vm_out = vc - 0.5 * slope;
    }

    /* one cell's 5-point (or 3-point) reconstruction along a direction */
    inline void recon1(const double *w, R (&v)[5], R &vm_out, R &vp_out) {
        int rc = cfg.recon;
        if (rc == CUMC_RECON_PPM) ppmc(w, v[0], v[1], v[2], v[3], v[4], vm_out, vp_out);
        else if (rc == CUMC_RECON_WENO) weno(w, v[0], v[1], v[2], v[3], v[4], vm_out, vp_out);
        else tvd(rc, w, v[1], v[2], v[3], vm_out, vp_out);
    }

    /* {TVD,PPMC,WENO}_recon{x,y,z}: tvd_module.f90:62-274,
     * ppmc_module.f90:151-352, weno_module.f90:154-308 */
    void recon(int dir) {
        int jl = 1, jh = nx, kl = 1, kh = ny, ll = 1, lh = nz;
        int dj = 0, dk = 0, dl = 0;
        int ibn, ibt1, ibt2;
        if (dir == x_dir) { jl = 0; jh = nx + 1; dj = 1; ibn = ibx; ibt1 = iby; ibt2 = ibz; }
        else if (dir == y_dir) { kl = 0; kh = ny + 1; dk = 1; ibn = iby; ibt1 = ibx; ibt2 = ibz; }
        else { ll = 0; lh = nz + 1; dl = 1; ibn = ibz; ibt1 = ibx; ibt2 = iby; }
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = ll; l <= lh; ++l)
            for (int k = kl; k <= kh; ++k)
                for (int j = jl; j <= jh; ++j) {
                    const double *w = (dir == x_dir) ? wx(j) : (dir == y_dir) ? wy(k) : wz(l);
                    int jm = j - dj, km = k - dk, lm = l - dl;
                    R v[5];
                    for (int i = imin; i <= itau; ++i) {
                        for (int s = -2; s <= 2; ++s) v[s + 2] = P(i, j + s * dj, k + s * dk, l + s * dl);
                        recon1(w, v, PR(i, jm, km, lm), PL(i, j, k, l));
                    }
                    /* optional positivity fallback (no counterpart in the reference):
                     * a cell whose reconstructed edge density or pressure is not
                     * positive is reconstructed at first order (edge = cell value) */
                    bool fallback = cfg.positivity_fallback &&
                        !(PR(irho, jm, km, lm) > 0.0 && PL(irho, j, k, l) > 0.0 &&
                          PR(itau, jm, km, lm) > 0.0 && PL(itau, j, k, l) > 0.0);
                    if (fallback) {
#pragma omp atomic
                        fb_count++;
                        for (int i = imin; i <= itau; ++i) { PR(i, jm, km, lm) = P(i, j, k, l); PL(i, j, k, l) = P(i, j, k, l); }
                    }
                    epsR[c3(jm, km, lm)] = eos_eps(PR(irho, jm, km, lm), PR(itau, jm, km, lm));
                    epsL[c3(j, k, l)] = eos_eps(PL(irho, j, k, l), PL(itau, j, k, l));
                    csR[c3(jm, km, lm)] = eos_cs(PR(itau, jm, km, lm), PR(irho, jm, km, lm), epsR[c3(jm, km, lm)]);
                    csL[c3(j, k, l)] = eos_cs(PL(itau, j, k, l), PL(irho, j, k, l), epsL[c3(j, k, l)]);
                    for (int i : {ibt1, ibt2}) {
                        for (int s = -2; s <= 2; ++s) v[s + 2] = BC(i, j + s * dj, k + s * dk, l + s * dl);
                        recon1(w, v, PR(i, jm, km, lm), PL(i, j, k, l));
                        if (fallback) { PR(i, jm, km, lm) = BC(i, j, k, l); PL(i, j, k, l) = BC(i, j, k, l); }
                    }
                    PR(ibn, jm, km, lm) = P(ibn, jm, km, lm);
                    PL(ibn, j, k, l) = P(ibn, j, k, l);
                }
    }

    /* ================================================================ */
    /* BUILDSTATES spatial.f90:272-403 (over the faces the solver reads) */
    /* ================================================================ */
    void dir_indices(int dir, int &ivn, int &ivt1, int &ivt2, int &ibn, int &ibt1, int &ibt2) {
        if (dir == x_dir) { ivn = ivx; ivt1 = ivy; ivt2 = ivz; ibn = ibx; ibt1 = iby; ibt2 = ibz; }
        else if (dir == y_dir) { ivn = ivy; ivt1 = ivz; ivt2 = ivx; ibn = iby; ibt1 = ibz; ibt2 = ibx; }
        else { ivn = ivz; ivt1 = ivx; ivt2 = ivy; ibn = ibz; ibt1 = ibx; ibt2 = iby; }
    }
    void face_range(int dir, int &jl, int &kl, int &ll) {
        jl = (dir == x_dir) ? 0 : 1; kl = (dir == y_dir) ? 0 : 1; ll = (dir == z_dir) ? 0 : 1;
    }

    void buildstates(int dir) {
        int ivn, ivt1, ivt2, ibn, ibt1, ibt2, jl, kl, ll;
        dir_indices(dir, ivn, ivt1, ivt2, ibn, ibt1, ibt2);
        face_range(dir, jl, kl, ll);
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = ll; l <= nz; ++l)
            for (int k = kl; k <= ny; ++k)
                for (int j = jl; j <= nx; ++j) {
                    for (int side = 0; side < 2; ++side) {
                        auto Pf = [&](int i) -> R & { return side == 0 ? PL(i, j, k, l) : PR(i, j, k, l); };
                        auto Uf = [&](int i) -> R & { return side == 0 ? UL(i, j, k, l) : URr(i, j, k, l); };
                        auto Ff = [&](int i) -> R & { return side == 0 ? FXL(i, j, k, l) : FXR(i, j, k, l); };
                        R ef = side == 0 ? epsL[c3(j, k, l)] : epsR[c3(j, k, l)];
                        R b2 = Pf(ibx) * Pf(ibx) + Pf(iby) * Pf(iby) + Pf(ibz) * Pf(ibz);
                        R v2 = Pf(ivx) * Pf(ivx) + Pf(ivy) * Pf(ivy) + Pf(ivz) * Pf(ivz);
                        R vb = Pf(ibx) * Pf(ivx) + Pf(iby) * Pf(ivy) + Pf(ibz) * Pf(ivz);
                        for (int i = imin; i <= itau; ++i) Uf(i) = Pf(i) * Pf(irho);
                        Uf(irho) = Pf(irho);
                        for (int i = ibx; i <= ibz; ++i) Uf(i) = Pf(i);
                        Uf(itau) = Pf(irho) * (0.5 * v2 + ef) + 0.5 * b2;
                        for (int i = imin; i <= itau; ++i) Ff(i) = Uf(i) * Pf(ivn);
                        Ff(ivn) = Ff(ivn) + Pf(itau) + 0.5 * (b2) - Pf(ibn) * Pf(ibn);
                        Ff(ivt1) = Ff(ivt1) - Pf(ibn) * Pf(ibt1);
                        Ff(ivt2) = Ff(ivt2) - Pf(ibn) * Pf(ibt2);
                        Ff(itau) = Ff(itau) + (Pf(itau) + 0.5 * (b2)) * Pf(ivn) - Pf(ibn) * vb;
                        Ff(ibn) = R(0.0);
                        Ff(ibt1) = (Pf(ivn) * Pf(ibt1) - Pf(ivt1) * Pf(ibn));
                        Ff(ibt2) = (Pf(ivn) * Pf(ibt2) - Pf(ivt2) * Pf(ibn));
                    }
                }
    }

    /* ================================================================ */
    /* Riemann solvers, rsolver_module.f90                              */
    /* ================================================================ */
    static R signalspeed(R cs_, R bn, R bt1, R bt2, R rho) { /* 32-48 */
        R a2 = cs_ * cs_;
        R a4 = a2 * a2;
        R b2n = (bn * bn / rho);
        R b2t1 = (bt1 * bt1 / rho);
        R b2t2 = (bt2 * bt2 / rho);
        R b2 = b2n + b2t1 + b2t2;
        R b4 = b2 * b2;
        return sqrt_(0.5 * (a2 + b2 + sqrt_(max_((a4 + b4 + 2.0 * b2 * a2) - 4.0 * a2 * b2n, R(0.0)))));
    }
    static R hll_state(R ul, R ur, R fl, R fr, R sl, R sr) { return (sr * ur - sl * ul - (fr - fl)) / (sr - sl); } /* 54-59 */
    static R hll_flux(R yl, R yr, R xl, R xr, R sl, R sr) { return (sr * yl - sl * yr + sl * sr * (xr - xl)) / (sr - sl); } /* 61-66 */
    static R roe(R xl, R xr, R rhol, R rhor) { return (sqrt_(rhol) * xl + sqrt_(rhor) * xr) / (sqrt_(rhol) + sqrt_(rhor)); } /* 68-73 */
    static R sstar_hllc(R pl, R pr, R rhol, R rhor, R vl, R vr, R sl, R sr, R bl, R br) { /* 86-93 */
        return (rhor * vr * (sr - vr) - rhol * vl * (sl - vl) + pl - pr + br * br - bl * bl) / (rhor * (sr - vr) - rhol * (sl - vl));
    }

    void riemann(int dir) {
        int ivn, ivt1, ivt2, ibn, ibt1, ibt2, jl, kl, ll;
        dir_indices(dir, ivn, ivt1, ivt2, ibn, ibt1, ibt2);
        face_range(dir, jl, kl, ll);
        const int rs = cfg.riemann;
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = ll; l <= nz; ++l)
            for (int k = kl; k <= ny; ++k)
                for (int j = jl; j <= nx; ++j) {
                    size_t c = c3(j, k, l);
                    R *pl = &primL[8 * c - 1], *pr = &primR[8 * c - 1]; /* 1-based */
                    R *ul = &uL[8 * c - 1], *ur = &uR[8 * c - 1];
                    R *fl = &fluxL[8 * c - 1], *fr = &fluxR[8 * c - 1];
                    R *fo = &flux[8 * c - 1];
                    R cfsL = signalspeed(csL[c], pl[ibn], pl[ibt1], pl[ibt2], pl[irho]);
                    R cfsR = signalspeed(csR[c], pr[ibn], pr[ibt1], pr[ibt2], pr[irho]);
                    if (rs == CUMC_RS_LF) { /* LFNM 133-222 */
                        R sL = abs_(pl[ivn]) + cfsL, sR = abs_(pr[ivn]) + cfsR;
                        R splus = max_(sL, sR);
                        for (int i = imin; i <= imax; ++i) fo[i] = 0.5 * (fl[i] + fr[i] - splus * (ur[i] - ul[i]));
                        continue;
                    }
                    R ubar = roe(pl[ivn], pr[ivn], pl[irho], pr[irho]);
                    R cbar = roe(cfsL, cfsR, pl[irho], pr[irho]);
                    R sL = min_(pl[ivn] - cfsL, ubar - cbar);
                    R sR = max_(pr[ivn] + cfsR, ubar + cbar);
                    if (rs == CUMC_RS_HLL) { /* HLLNM 227-326 */
                        if (sL >= 0.0) { for (int i = imin; i <= imax; ++i) fo[i] = fl[i]; }
                        else if (sL <= 0.0 && sR >= 0.0) { for (int i = imin; i <= imax; ++i) fo[i] = hll_flux(fl[i], fr[i], ul[i], ur[i], sL, sR); }
                        else if (sR <= 0.0) { for (int i = imin; i <= imax; ++i) fo[i] = fr[i]; }
                        continue;
                    }
                    if (sL >= 0.0) { for (int i = imin; i <= imax; ++i) fo[i] = fl[i]; continue; }
                    if (sR <= 0.0) { for (int i = imin; i <= imax; ++i) fo[i] = fr[i]; continue; }
                    R b2L = pl[ibx] * pl[ibx] + pl[iby] * pl[iby] + pl[ibz] * pl[ibz];
                    R b2R = pr[ibx] * pr[ibx] + pr[iby] * pr[iby] + pr[ibz] * pr[ibz];
                    R pLt = pl[itau] + 0.5 * b2L;
                    R pRt = pr[itau] + 0.5 * b2R;
                    if (rs == CUMC_RS_HLLC) hllc_star(pl, pr, ul, ur, fl, fr, fo, sL, sR, pLt, pRt, ivn, ivt1, ivt2, ibn, ibt1, ibt2);
                    else hlld_star(pl, pr, ul, ur, fl, fr, fo, sL, sR, pLt, pRt, ivn, ivt1, ivt2, ibn, ibt1, ibt2);
                }
    }

    /* HLLCNM star region, rsolver_module.f90:423-498 */
    static void hllc_star(R *pl, R *pr, R *ul, R *ur, R *fl, R *fr, R *fo, R sL, R sR, R pLt, R pRt,
                          int ivn, int ivt1, int ivt2, int ibn, int ibt1, int ibt2) {
        R u_hll[9], p_hll[9], us[9];
        R sstar = sstar_hllc(pLt, pRt, pl[irho], pr[irho], pl[ivn], pr[ivn], sL, sR, pl[ibn], pr[ibn]);
        u_hll[ibn] = pl[ibn];
        u_hll[ibt1] = hll_state(pl[ibt1], pr[ibt1], fl[ibt1], fr[ibt1], sL, sR);
        u_hll[ibt2] = hll_state(pl[ibt2], pr[ibt2], fl[ibt2], fr[ibt2], sL, sR);
        u_hll[irho] = hll_state(pl[irho], pr[irho], fl[irho], fr[irho], sL, sR);
        u_hll[ivt1] = hll_state(ul[ivt1], ur[ivt1], fl[ivt1], fr[ivt1], sL, sR);
        u_hll[ivt2] = hll_state(ul[ivt2], ur[ivt2], fl[ivt2], fr[ivt2], sL, sR);
        p_hll[ivn] = sstar;
        p_hll[ivt1] = u_hll[ivt1] / u_hll[irho];
        p_hll[ivt2] = u_hll[ivt2] / u_hll[irho];
        const bool left = (sstar >= 0.0);
        R *pS = left ? pl : pr, *uS = left ? ul : ur, *fS = left ? fl : fr;
        R s = left ? sL : sR, pSt = left ? pLt : pRt;
        us[irho] = uS[irho] * (s - pS[ivn]) / (s - sstar);
        R vb = pS[ibx] * pS[ivx] + pS[iby] * pS[ivy] + pS[ibz] * pS[ivz];
        R vbhll = u_hll[ibx] * p_hll[ivx] + u_hll[iby] * p_hll[ivy] + u_hll[ibz] * p_hll[ivz];
        R ps = pS[irho] * (s - pS[ivn]) * (sstar - pS[ivn]) + pSt;
        us[ibn] = u_hll[ibn];
        us[ibt1] = u_hll[ibt1];
        us[ibt2] = u_hll[ibt2];
        us[ivn] = us[irho] * sstar;
        us[ivt1] = (uS[ivt1] * (s - pS[ivn]) - (us[ibn] * us[ibt1] - pS[ibn] * pS[ibt1])) / (s - sstar);
        us[ivt2] = (uS[ivt2] * (s - pS[ivn]) - (us[ibn] * us[ibt2] - pS[ibn] * pS[ibt2])) / (s - sstar);
        us[itau] = (uS[itau] * (s - pS[ivn]) + (ps * sstar - pSt * pS[ivn]) - ((vbhll * us[ibn] - vb * pS[ibn]))) / (s - sstar);
        for (int i = imin; i <= imax; ++i) fo[i] = fS[i] + s * (us[i] - uS[i]);
    }

    /* HLLDNM star / double-star regions, rsolver_module.f90:613-750.
     * The reference never assigns the normal component of the double-star
     * states (usstarL/usstarR(ibn)); those PRIVATE arrays then hold undefined
     * values.  Here they take the HLLD value B_n (Miyoshi & Kusano 2005:
     * B_x is constant across the fan), i.e. usstar(ibn) = ustar(ibn). */
    static void hlld_star(R *pl, R *pr, R *ul, R *ur, R *fl, R *fr, R *fo, R sL, R sR, R pLt, R pRt,
                          int ivn, int ivt1, int ivt2, int ibn, int ibt1, int ibt2) {
        R usL[9], usR[9], pstL[9], pstR[9], ussL[9], ussR[9], pssL[9], pssR[9];
        R sM = sstar_hllc(pLt, pRt, pl[irho], pr[irho], pl[ivn], pr[ivn], sL, sR, pl[ibn], pr[ibn]);
        for (int i = irho; i <= itau; ++i) usL[i] = ul[i] * (sL - pl[ivn]) / (sL - sM);
        for (int i = irho; i <= itau; ++i) usR[i] = ur[i] * (sR - pr[ivn]) / (sR - sM);
        R sstarL = sM - abs_(pl[ibn]) / sqrt_(usL[irho]);
        R sstarR = sM + abs_(pr[ibn]) / sqrt_(usR[irho]);
        if (((sstarL - sL) < 1.0e-4 * (sM - sL)) || ((sstarR - sR) > -1.0e-4 * (sR - sM))) {
            usL[ibn] = pl[ibn];
            usL[ibt1] = hll_state(pl[ibt1], pr[ibt1], fl[ibt1], fr[ibt1], sL, sR);
            usL[ibt2] = hll_state(pl[ibt2], pr[ibt2], fl[ibt2], fr[ibt2], sL, sR);
            usR[ibn] = pr[ibn];
            usR[ibt1] = usL[ibt1];
            usR[ibt2] = usL[ibt2];
            sstarL = sM;
            sstarR = sM;
        } else {
            R fac_1 = (pl[irho] * (sL - pl[ivn]) * (sL - sM) - pl[ibn] * pl[ibn]);
            usL[ibn] = pl[ibn];
            usL[ibt1] = (pl[ibt1] * (pl[irho] * (sL - pl[ivn]) * (sL - pl[ivn]) - pl[ibn] * pl[ibn])) / fac_1;
            usL[ibt2] = (pl[ibt2] * (pl[irho] * (sL - pl[ivn]) * (sL - pl[ivn]) - pl[ibn] * pl[ibn])) / fac_1;
            fac_1 = (pr[irho] * (sR - pr[ivn]) * (sR - sM) - pr[ibn] * pr[ibn]);
            usR[ibn] = pr[ibn];
            usR[ibt1] = (pr[ibt1] * (pr[irho] * (sR - pr[ivn]) * (sR - pr[ivn]) - pr[ibn] * pr[ibn])) / fac_1;
            usR[ibt2] = (pr[ibt2] * (pr[irho] * (sR - pr[ivn]) * (sR - pr[ivn]) - pr[ibn] * pr[ibn])) / fac_1;
        }
        usL[ivn] = usL[irho] * sM;
        usL[ivt1] = usL[ivt1] - (usL[ibn] * usL[ibt1] - pl[ibn] * pl[ibt1]) / (sL - sM);
        usL[ivt2] = usL[ivt2] - (usL[ibn] * usL[ibt2] - pl[ibn] * pl[ibt2]) / (sL - sM);
        usR[ivn] = usR[irho] * sM;
        usR[ivt1] = usR[ivt1] - (usR[ibn] * usR[ibt1] - pr[ibn] * pr[ibt1]) / (sR - sM);
        usR[ivt2] = usR[ivt2] - (usR[ibn] * usR[ibt2] - pr[ibn] * pr[ibt2]) / (sR - sM);
        pstL[ivn] = sM;
        pstL[ivt1] = usL[ivt1] / usL[irho];
        pstL[ivt2] = usL[ivt2] / usL[irho];
        pstR[ivn] = sM;
        pstR[ivt1] = usR[ivt1] / usR[irho];
        pstR[ivt2] = usR[ivt2] / usR[irho];
        R pLs = pl[irho] * (sL - pl[ivn]) * (sM - pl[ivn]) + pLt;
        R pRs = pr[irho] * (sR - pr[ivn]) * (sM - pr[ivn]) + pRt;
        R bdotu = pl[ibx] * pl[ivx] + pl[iby] * pl[ivy] + pl[ibz] * pl[ivz];
        R bdotus = usL[ibx] * pstL[ivx] + usL[iby] * pstL[ivy] + usL[ibz] * pstL[ivz];
        usL[itau] = usL[itau] + ((pLs * sM - pLt * pl[ivn]) - (bdotus - bdotu) * pl[ibn]) / (sL - sM);
        bdotu = pr[ibx] * pr[ivx] + pr[iby] * pr[ivy] + pr[ibz] * pr[ivz];
        bdotus = usR[ibx] * pstR[ivx] + usR[iby] * pstR[ivy] + usR[ibz] * pstR[ivz];
        usR[itau] = usR[itau] + ((pRs * sM - pRt * pr[ivn]) - (bdotus - bdotu) * pr[ibn]) / (sR - sM);
        if (sstarL >= 0.0) {
            for (int i = imin; i <= imax; ++i) fo[i] = fl[i] + sL * (usL[i] - ul[i]);
        } else if (sstarR <= 0.0) {
            for (int i = imin; i <= imax; ++i) fo[i] = fr[i] + sR * (usR[i] - ur[i]);
        } else {
            ussL[irho] = usL[irho];
            ussR[irho] = usR[irho];
            R fac_1 = 1.0 / (sqrt_(usL[irho]) + sqrt_(usR[irho]));
            R fac_2 = sign1_(pl[ibn]);
            pssL[ivn] = sM;
            pssL[ivt1] = fac_1 * (sqrt_(usL[irho]) * pstL[ivt1] + sqrt_(usR[irho]) * pstR[ivt1] + (usR[ibt1] - usL[ibt1]) * fac_2);
            pssL[ivt2] = fac_1 * (sqrt_(usL[irho]) * pstL[ivt2] + sqrt_(usR[irho]) * pstR[ivt2] + (usR[ibt2] - usL[ibt2]) * fac_2);
            ussL[ibt1] = fac_1 * (sqrt_(usL[irho]) * usR[ibt1] + sqrt_(usR[irho]) * usL[ibt1] + sqrt_(usL[irho] * usR[irho]) * (pstR[ivt1] - pstL[ivt1]) * fac_2);
            ussL[ibt2] = fac_1 * (sqrt_(usL[irho]) * usR[ibt2] + sqrt_(usR[irho]) * usL[ibt2] + sqrt_(usL[irho] * usR[irho]) * (pstR[ivt2] - pstL[ivt2]) * fac_2);
            ussL[ibn] = usL[ibn];
            ussL[ivn] = ussL[irho] * pssL[ivn];
            ussL[ivt1] = ussL[irho] * pssL[ivt1];
            ussL[ivt2] = ussL[irho] * pssL[ivt2];
            bdotus = usL[ibx] * pstL[ivx] + usL[iby] * pstL[ivy] + usL[ibz] * pstL[ivz];
            R bdotuss = ussL[ibx] * pssL[ivx] + ussL[iby] * pssL[ivy] + ussL[ibz] * pssL[ivz];
            ussL[itau] = usL[itau] - sqrt_(usL[irho]) * (bdotus - bdotuss) * fac_2;
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
            ussR[itau] = usR[itau] + sqrt_(usR[irho]) * (bdotus - bdotuss) * fac_2;
            if (sM >= 0.0) {
                for (int i = imin; i <= imax; ++i) fo[i] = fl[i] + sL * (usL[i] - ul[i]) + sstarL * (ussL[i] - usL[i]);
            } else {
                for (int i = imin; i <= imax; ++i) fo[i] = fr[i] + sR * (usR[i] - ur[i]) + sstarR * (ussR[i] - usR[i]);
            }
        }
    }

    /* ================================================================ */
    /* SPATIAL pieces                                                   */
    /* ================================================================ */
    /* GET_SOURCE spatial.f90:167-267 */
    void get_source() {
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    for (int i = imin; i <= imax; ++i) SC(i, j, k, l) = R(0.0);
                    if (coord == 0) continue;
                    R bx = BC(ibx, j, k, l), by = BC(iby, j, k, l), bz = BC(ibz, j, k, l);
                    R rho = P(irho, j, k, l), vx = P(ivx, j, k, l), vy = P(ivy, j, k, l), vz = P(ivz, j, k, l), p = P(itau, j, k, l);
                    R bsquare = bx * bx + by * by + bz * bz;
                    if (coord == 1) {
                        SC(ivx, j, k, l) = SC(ivx, j, k, l) + (p + rho * vy * vy + 0.5 * bsquare - by * by) / (x(j));
                        SC(ivy, j, k, l) = SC(ivy, j, k, l) - (rho * vx * vy - bx * by) / (x(j));
                    } else {
                        R G = R(3.0 * x(j) * dx(j) / dx_cb(j));
                        R tf = R(dsine(k) / dcose(k));
                        SC(ivx, j, k, l) = SC(ivx, j, k, l) + (2.0 * p + bx * bx + rho * (vy * vy + vz * vz)) * G;
                        SC(ivy, j, k, l) = SC(ivy, j, k, l) + (p + rho * vz * vz + 0.5 * bsquare - bz * bz) * G * tf
                                           - (rho * vx * vy - bx * by) * G;
                        SC(ivz, j, k, l) = SC(ivz, j, k, l) - (rho * vx * vz - bx * bz) * G
                                           - (rho * vy * vz - by * bz) * G * tf;
                    }
                }
    }

    /* FLUX_DIFF spatial.f90:408-592 */
    void flux_diff(int dir) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j)
                    for (int i = imin; i <= itau; ++i) {
                        R dflux;
                        if (dir == x_dir) {
                            if (coord == 0) dflux = (FL(i, j, k, l) - FL(i, j - 1, k, l)) / (dx(j));
                            else if (coord == 1) dflux = (xF(j) * FL(i, j, k, l) - xF(j - 1) * FL(i, j - 1, k, l)) / (x(j) * dx(j));
                            else dflux = (xF(j) * xF(j) * FL(i, j, k, l) - xF(j - 1) * xF(j - 1) * FL(i, j - 1, k, l)) / (dx_cb(j) / 3.0);
                            LR(i, j, k, l) = -dflux;
                        } else if (dir == y_dir) {
                            if (coord == 0) dflux = (FL(i, j, k, l) - FL(i, j, k - 1, l)) / (dy(k));
                            else if (coord == 1) dflux = (FL(i, j, k, l) - FL(i, j, k - 1, l)) / (x(j) * dy(k));
                            else dflux = (sinf(k) * FL(i, j, k, l) - sinf(k - 1) * FL(i, j, k - 1, l)) / (xbar(j) * dcose(k));
                            LR(i, j, k, l) = LR(i, j, k, l) - dflux;
                        } else {
                            if (coord == 0 || coord == 1) dflux = (FL(i, j, k, l) - FL(i, j, k, l - 1)) / dz(l);
                            else dflux = (FL(i, j, k, l) - FL(i, j, k, l - 1)) * dy(k) / (xbar(j) * dz(l) * dcose(k));
                            LR(i, j, k, l) = LR(i, j, k, l) - dflux;
                        }
                    }
    }

    /* MHD_FLUX mhd_module.f90:206-280 */
    void mhd_flux(int dir) {
        int jl, kl, ll;
        face_range(dir, jl, kl, ll);
        for (int l = ll; l <= nz; ++l)
            for (int k = kl; k <= ny; ++k)
                for (int j = jl; j <= nx; ++j) {
                    if (dir == x_dir) { EF(iyx, j, k, l) = FL(ibz, j, k, l); EF(izx, j, k, l) = -FL(iby, j, k, l); }
                    else if (dir == y_dir) { EF(ixy, j, k, l) = -FL(ibz, j, k, l); EF(izy, j, k, l) = FL(ibx, j, k, l); }
                    else { EF(ixz, j, k, l) = FL(iby, j, k, l); EF(iyz, j, k, l) = -FL(ibx, j, k, l); }
                }
    }

    /* BOUNDARY_EFIELD mhd_module.f90:478-840 */
    void boundary_efield() {
        auto ecv = [&](int i) { return [this, i](int j, int k, int l) -> R & { return EC(i, j, k, l); }; };
        auto efv = [&](int i) { return [this, i](int j, int k, int l) -> R & { return EF(i, j, k, l); }; };
        for (int i = iex; i <= iez; ++i) fill_x(ecv(i), bfac_xin[i], bfac_xout[i]);
        fill_x(efv(ixz), bfac_xin[iex], bfac_xout[iex]);
        fill_x(efv(ixy), bfac_xin[iex], bfac_xout[iex]);
        fill_x(efv(iyz), bfac_xin[iey], bfac_xout[iey]);
        fill_x(efv(izy), bfac_xin[iez], bfac_xout[iez]);
        for (int i = iex; i <= iez; ++i) fill_y(ecv(i), bfac_yin[i], bfac_yout[i], false);
        fill_y(efv(ixz), bfac_yin[iex], bfac_yout[iex], false);
        fill_y(efv(iyx), bfac_yin[iey], bfac_yout[iey], false);
        fill_y(efv(iyz), bfac_yin[iey], bfac_yout[iey], false);
        fill_y(efv(izx), bfac_yin[iez], bfac_yout[iez], false);
        for (int i = iex; i <= iez; ++i) fill_z(ecv(i), bfac_zin[i], bfac_zout[i]);
        fill_z(efv(ixy), bfac_zin[iex], bfac_zout[iex]);
        fill_z(efv(iyx), bfac_zin[iey], bfac_zout[iey]);
        fill_z(efv(izx), bfac_zin[iez], bfac_zout[iez]);
        fill_z(efv(izy), bfac_zin[iez], bfac_zout[iez]);
    }

    /* flux_ct mhd_module.f90:285-473 */
    void flux_ct() {
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    EC(iex, j, k, l) = P(ivz, j, k, l) * BC(iby, j, k, l) - P(ivy, j, k, l) * BC(ibz, j, k, l);
                    EC(iey, j, k, l) = P(ivx, j, k, l) * BC(ibz, j, k, l) - P(ivz, j, k, l) * BC(ibx, j, k, l);
                    EC(iez, j, k, l) = P(ivy, j, k, l) * BC(ibx, j, k, l) - P(ivx, j, k, l) * BC(iby, j, k, l);
                }
        if (n_dim == 1) {
            for (int j = 1; j <= nx; ++j) {
                EF(ixy, j, 1, 1) = EC(iex, j, 1, 1);
                EF(izy, j, 1, 1) = EC(iez, j, 1, 1);
                EF(ixy, j, 0, 1) = EC(iex, j, 1, 1);
                EF(izy, j, 0, 1) = EC(iez, j, 1, 1);
                EF(ixz, j, 1, 1) = EC(iex, j, 1, 1);
                EF(iyz, j, 1, 1) = EC(iey, j, 1, 1);
                EF(ixz, j, 1, 0) = EC(iex, j, 1, 1);
                EF(iyz, j, 1, 0) = EC(iey, j, 1, 1);
            }
        } else if (n_dim == 2) {
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    EF(ixz, j, k, 1) = EC(iex, j, k, 1);
                    EF(iyz, j, k, 1) = EC(iey, j, k, 1);
                    EF(ixz, j, k, 0) = EC(iex, j, k, 1);
                    EF(iyz, j, k, 0) = EC(iey, j, k, 1);
                }
        }
        boundary_efield();
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    EX(j, k, l) = 0.50 * (EF(ixy, j, k, l) + EF(ixy, j, k, l + 1) + EF(ixz, j, k, l) + EF(ixz, j, k + 1, l))
                                  - 0.25 * (EC(iex, j, k, l) + EC(iex, j, k, l + 1) + EC(iex, j, k + 1, l) + EC(iex, j, k + 1, l + 1));
                    EY(j, k, l) = 0.50 * (EF(iyx, j, k, l) + EF(iyx, j, k, l + 1) + EF(iyz, j, k, l) + EF(iyz, j + 1, k, l))
                                  - 0.25 * (EC(iey, j, k, l) + EC(iey, j, k, l + 1) + EC(iey, j + 1, k, l) + EC(iey, j + 1, k, l + 1));
                    EZ(j, k, l) = 0.50 * (EF(izx, j, k, l) + EF(izx, j, k + 1, l) + EF(izy, j, k, l) + EF(izy, j + 1, k, l))
                                  - 0.25 * (EC(iez, j, k, l) + EC(iez, j, k + 1, l) + EC(iez, j + 1, k, l) + EC(iez, j + 1, k + 1, l));
                }
        if (cfg.fixpole && coord == 2) {
            /* mhd_module.f90:437-461: REAL (single precision) accumulators */
            for (int j = 1; j <= nx; ++j) {
                float sum1 = 0.0f, sum2 = 0.0f;
                for (int l = 1; l <= nz; ++l) {
                    sum1 = (float)((double)sum1 + dv(EX(j, 0, l)));
                    sum2 = (float)((double)sum2 + dv(EX(j, ny, l)));
                }
                for (int l = -2; l <= nz + 3; ++l) {
                    EX(j, 0, l) = R((double)sum1 / (double)nz);
                    EX(j, ny, l) = R((double)sum2 / (double)nz);
                }
            }
        }
    }

    /* l_operator spatial.f90:597-713 */
    void l_operator() {
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j)
                    for (int i = imin; i <= itau; ++i) LR(i, j, k, l) = LR(i, j, k, l) + SC(i, j, k, l);
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j) {
                    if (coord == 0) {
                        LR(ibx, j, k, l) = -((EZ(j, k, l) - EZ(j, k - 1, l)) / (dy(k)) - (EY(j, k, l) - EY(j, k, l - 1)) / (dz(l)));
                        LR(iby, j, k, l) = -((EX(j, k, l) - EX(j, k, l - 1)) / (dz(l)) - (EZ(j, k, l) - EZ(j - 1, k, l)) / (dx(j)));
                        LR(ibz, j, k, l) = -((EY(j, k, l) - EY(j - 1, k, l)) / (dx(j)) - (EX(j, k, l) - EX(j, k - 1, l)) / (dy(k)));
                    } else if (coord == 1) {
                        LR(ibx, j, k, l) = -(EZ(j, k, l) - EZ(j, k - 1, l)) / (xF(j) * dy(k)) + (EY(j, k, l) - EY(j, k, l - 1)) / (dz(l));
                        LR(iby, j, k, l) = -(EX(j, k, l) - EX(j, k, l - 1)) / (dz(l)) + (EZ(j, k, l) - EZ(j - 1, k, l)) / (dx(j));
                        LR(ibz, j, k, l) = -(xF(j) * EY(j, k, l) - xF(j - 1) * EY(j - 1, k, l)) / (x(j) * dx(j)) + (EX(j, k, l) - EX(j, k - 1, l)) / (x(j) * dy(k));
                    } else {
                        LR(ibx, j, k, l) = (-(sinf(k) * EZ(j, k, l) - sinf(k - 1) * EZ(j, k - 1, l)) + (EY(j, k, l) - EY(j, k, l - 1)) * (dy(k) / dz(l))) / (xF(j) * dcose(k) + small_num);
                        LR(iby, j, k, l) = (-(EX(j, k, l) - EX(j, k, l - 1)) / (xbar(j) * sinf(k) * dz(l) + small_num) + (xF(j) * EZ(j, k, l) - xF(j - 1) * EZ(j - 1, k, l)) / (x(j) * dx(j)));
                        LR(ibz, j, k, l) = (-(xF(j) * EY(j, k, l) - xF(j - 1) * EY(j - 1, k, l)) / (x(j) * dx(j)) + (EX(j, k, l) - EX(j, k - 1, l)) / (xbar(j) * dy(k)));
                    }
                }
    }

    /* SPATIAL spatial.f90:11-162 */
    void spatial() {
        get_source();
        custom_source();
        for (int dir = 1; dir <= n_dim; ++dir) {
            {
                PhaseScope ph(PH_RECON);
                recon(dir);
            }
            {
                PhaseScope ph(PH_RIEMANN);
                buildstates(dir);
                riemann(dir);
            }
            if (dir == 1 && cfg.model.source_kind == CUMC_SRC_COLLAPSAR) {
                /* GETFLUX_X, model/collapsar/src/custom.f90:222-240 */
                mflux.assign((size_t)ny * nz, R(0.0));
                for (int l = 1; l <= nz; ++l)
                    for (int k = 1; k <= ny; ++k) mflux[(size_t)(k - 1) + (size_t)ny * (l - 1)] = FL(irho, 0, k, l);
            }
            flux_diff(dir);
            mhd_flux(dir);
        }
        flux_ct();
        l_operator();
    }

    /* ================================================================ */
    /* time integration, rungekutta.f90                                 */
    /* ================================================================ */
    void rk_combine(int stage, double dt) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j)
                    for (int i = imin; i <= imax; ++i) {
                        /* the reference's l_rk is undefined for hydro at index 0
                         * (spatial.f90:440-449 fills 1..n); zero it here */
                        bool ghost0 = (j == 0 || k == 0 || l == 0);
                        R lr = (ghost0 && i < ibx) ? R(0.0) : LR(i, j, k, l);
                        if (stage == 1) U(i, j, k, l) = UO(i, j, k, l) + dt * lr;
                        else if (stage == 2) U(i, j, k, l) = rk20 * UO(i, j, k, l) + rk21 * U(i, j, k, l) + rk22 * dt * lr;
                        else U(i, j, k, l) = rk30 * UO(i, j, k, l) + rk31 * U(i, j, k, l) + rk32 * dt * lr;
                    }
    }

    /* RUNGEKUTTA rungekutta.f90:12-208 */
    void rungekutta(double dt) {
#pragma omp parallel for collapse(2) schedule(static)
        for (int l = 0; l <= nz; ++l)
            for (int k = 0; k <= ny; ++k)
                for (int j = 0; j <= nx; ++j)
                    for (int i = imin; i <= imax; ++i) UO(i, j, k, l) = U(i, j, k, l);
        for (int stage = 1; stage <= 3; ++stage) {
            spatial();
            rk_combine(stage, dt);
            fromutorve();
            custom_checkrho();
            if (stage == 3) custom_checkrho(); /* OPERATOR_SPLIT is empty */
            fromrvetou();
            boundary();
            update();
            custom_update(stage, dt);
        }
    }

    /* CUSTOM_UPDATE of the collapsar model for p_in = stage > 0
     * (model/collapsar/src/custom.f90:450-485): mdot from the inner-face mass
     * flux, the black hole mass by the stage's Shu-Osher weights, r_sh.  The
     * reference sums with an OpenMP reduction of unspecified order; this
     * sums in the engine's fixed order: 1024 strided partial sums, each in
     * sequence, then a pairwise tree. */
    void custom_update(int stage, double dt) {
        if (cfg.model.source_kind != CUMC_SRC_COLLAPSAR) return;
        const int n = ny * nz;
        std::vector<R> part(1024);
        const double xf0 = xF(0);
        for (int t = 0; t < 1024; ++t) {
            R acc = R(0.0);
            for (int i = t; i < n; i += 1024) {
                const int k = i % ny + 1, l = i / ny + 1;
                acc = acc + (-mflux[(size_t)i]) * xf0 * xf0 * dcose(k) * dz(l);
            }
            part[(size_t)t] = acc;
        }
        for (int s = 512; s > 0; s >>= 1)
            for (int t = 0; t < s; ++t) part[(size_t)t] = part[(size_t)t] + part[(size_t)(t + s)];
        const double mdot = dv(max_(part[0], R(0.0)));
        if (stage == 1) {
            mbh_old = m_bh;
            m_bh = mbh_old + dt * mdot;
        } else if (stage == 2) {
            m_bh = rk20 * mbh_old + rk21 * m_bh + rk22 * dt * mdot;
        } else {
            m_bh = rk30 * mbh_old + rk31 * m_bh + rk32 * dt * mdot;
        }
        r_sh = 2.0 * m_bh / (c_code * c_code);
        if (r_sh >= xf0) horizon_hit = true;  /* the reference STOPs */
    }

    /* INITIAL_UPDATE initial.f90:86-116 */
    void initial_update() {
        custom_checkrho();
        fromrvetou();
        boundary();
        update();
    }

    /* FINDDT rungekutta.f90:221-332 */
    double finddt() {
        PhaseScope ph(PH_DT);
        double dt_out2 = 1.0e5;
#pragma omp parallel for collapse(2) schedule(static) reduction(min : dt_out2)
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    R rho = P(irho, j, k, l);
                    R a2 = CS(j, k, l) * CS(j, k, l);
                    R a4 = a2 * a2;
                    R b2x = (BC(ibx, j, k, l) * BC(ibx, j, k, l) / rho);
                    R b2y = (BC(iby, j, k, l) * BC(iby, j, k, l) / rho);
                    R b2z = (BC(ibz, j, k, l) * BC(ibz, j, k, l) / rho);
                    R b2 = b2x + b2y + b2z;
                    R b4 = b2 * b2;
                    R cfx = sqrt_(0.5 * (a2 + b2 + sqrt_((a4 + 2.0 * a2 * b2 + b4) - 4.0 * a2 * b2x)));
                    R cfy = sqrt_(0.5 * (a2 + b2 + sqrt_((a4 + 2.0 * a2 * b2 + b4) - 4.0 * a2 * b2y)));
                    R cfz = sqrt_(0.5 * (a2 + b2 + sqrt_((a4 + 2.0 * a2 * b2 + b4) - 4.0 * a2 * b2z)));
                    R lambda1 = abs_(P(ivx, j, k, l)) + cfx;
                    R lambda2 = abs_(P(ivy, j, k, l)) + cfy;
                    R lambda3 = abs_(P(ivz, j, k, l)) + cfz;
                    R lambda = max3_(lambda1, lambda2, lambda3);
                    R dtt = R(dx(j));
                    if (coord == 0) {
                        if (n_dim > 1) dtt = min_(dtt, R(dy(k)));
                        if (n_dim > 2) dtt = min_(dtt, R(dz(l)));
                    } else if (coord == 1) {
                        if (n_dim > 1 && ny > 1) dtt = min_(dtt, R(x(j) * dy(k)));
                        if (n_dim > 2) dtt = min_(dtt, R(dz(l)));
                    } else {
                        if (n_dim > 1) dtt = min_(dtt, R(x(j) * dy(k)));
                        if (n_dim > 2) dtt = min_(dtt, R(x(j) * sine(k) * dz(l)));
                    }
                    dtt = dtt * cfl / lambda;
                    double d = dv(dtt);
                    if (d < dt_out2) dt_out2 = d;
                }
        return std::min(1.0e5, dt_out2);
    }

    /* FIND_DIVB mhd_module.f90:110-201 */
    double find_divb() {
        double m = 0.0;
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    double d;
                    double bx = dv(P(ibx, j, k, l)), bxm = dv(P(ibx, j - 1, k, l));
                    double by = dv(P(iby, j, k, l)), bym = dv(P(iby, j, k - 1, l));
                    double bz = dv(P(ibz, j, k, l)), bzm = dv(P(ibz, j, k, l - 1));
                    if (coord == 0)
                        d = (bx - bxm) / (dx(j)) + (by - bym) / (dy(k)) + (bz - bzm) / (dz(l));
                    else if (coord == 1)
                        d = (xF(j) * bx - xF(j - 1) * bxm) / (x(j) * dx(j)) + (by - bym) / (x(j) * dy(k)) + (bz - bzm) / (dz(l));
                    else
                        d = (xF(j) * xF(j) * bx - xF(j - 1) * xF(j - 1) * bxm) / (dx_cb(j) / 3.0)
                            + (sinf(k) * by - sinf(k - 1) * bym) * (x(j) * dx(j)) / (dx_cb(j) * dcose(k) / 3.0)
                            + (bz - bzm) * (x(j) * dx(j) * dy(k)) / (dx_cb(j) * dcose(k) * dz(l) / 3.0);
                    m = std::max(m, std::fabs(d));
                }
        return m;
    }
};

/* ------------------------------------------------------------------ */
/* C API (used by tests, smoke and the bench baselines only)           */
/* ------------------------------------------------------------------ */
struct Handle {
    int counting;
    Sim<double> *d = nullptr;
    Sim<CReal> *c = nullptr;
    std::string err;
};

static std::string g_err;

/* the operation counters are plain globals: counting runs use one thread */
struct SerialScope {
    int saved = 1;
    bool on;
    explicit SerialScope(bool c) : on(c) {
#ifdef _OPENMP
        if (on) { saved = omp_get_max_threads(); omp_set_num_threads(1); }
#endif
    }
    ~SerialScope() {
#ifdef _OPENMP
        if (on) omp_set_num_threads(saved);
#endif
    }
};

} // namespace orc

using namespace orc;

template <class R>
static void set_state_t(Sim<R> *s, const double *prim, const double *eps) {
    size_t n3 = (size_t)s->NX * s->NY * s->NZ;
    for (size_t i = 0; i < 8 * n3; ++i) s->prim[i] = R(prim[i]);
    for (size_t i = 0; i < n3; ++i) s->eps[i] = R(eps[i]);
}
template <class R>
static void get_state_t(Sim<R> *s, double *prim, double *eps) {
    size_t n3 = (size_t)s->NX * s->NY * s->NZ;
    for (size_t i = 0; i < 8 * n3; ++i) prim[i] = dv(s->prim[i]);
    for (size_t i = 0; i < n3; ++i) eps[i] = dv(s->eps[i]);
}

extern "C" {

void *orc_create(const cumc_config *cfg, int counting) {
    Handle *h = new Handle();
    h->counting = counting;
    int rc;
    if (counting) { h->c = new Sim<CReal>(); rc = h->c->init(cfg); if (rc) g_err = h->c->err; }
    else { h->d = new Sim<double>(); rc = h->d->init(cfg); if (rc) g_err = h->d->err; }
    if (rc) { delete h->c; delete h->d; delete h; return nullptr; }
    return h;
}
const char *orc_last_error(void) { return g_err.c_str(); }

void orc_destroy(void *p) {
    Handle *h = (Handle *)p;
    if (!h) return;
    delete h->c; delete h->d; delete h;
}

void orc_set_state(void *p, const double *prim, const double *eps) {
    Handle *h = (Handle *)p;
    if (h->counting) set_state_t(h->c, prim, eps); else set_state_t(h->d, prim, eps);
}
void orc_get_state(void *p, double *prim, double *eps) {
    Handle *h = (Handle *)p;
    if (h->counting) get_state_t(h->c, prim, eps); else get_state_t(h->d, prim, eps);
}
/* which: 0 cons, 1 bcell, 2 cs */
void orc_get_array(void *p, int which, double *out) {
    Handle *h = (Handle *)p;
    auto grab = [&](auto *s) {
        size_t n3 = (size_t)s->NX * s->NY * s->NZ;
        if (which == 0) for (size_t i = 0; i < 8 * n3; ++i) out[i] = dv(s->cons[i]);
        else if (which == 1) for (size_t i = 0; i < 3 * n3; ++i) out[i] = dv(s->bcell[i]);
        else if (which == 2) for (size_t i = 0; i < n3; ++i) out[i] = dv(s->cs[i]);
    };
    if (h->counting) grab(h->c); else grab(h->d);
}
unsigned long long orc_fallback_count(void *p) {
    Handle *h = (Handle *)p;
    return h->counting ? h->c->fb_count : h->d->fb_count;
}
void orc_initial_update(void *p) {
    SerialScope serial_(((Handle *)p)->counting != 0);
    Handle *h = (Handle *)p;
    if (h->counting) h->c->initial_update(); else h->d->initial_update();
}
double orc_finddt(void *p) {
    SerialScope serial_(((Handle *)p)->counting != 0);
    Handle *h = (Handle *)p;
    return h->counting ? h->c->finddt() : h->d->finddt();
}
void orc_rk3_step(void *p, double dt) {
    SerialScope serial_(((Handle *)p)->counting != 0);
    Handle *h = (Handle *)p;
    if (h->counting) h->c->rungekutta(dt); else h->d->rungekutta(dt);
}
/* main.f90:98-139 loop; returns the number of steps */
int orc_evolve(void *p, double t_end, int max_steps, double *t_inout) {
    Handle *h = (Handle *)p;
    double t = *t_inout;
    int n = 0;
    while (t < t_end && n < max_steps) {
        double dt = orc_finddt(p);
        if (t + dt > t_end) dt = t_end - t;
        orc_rk3_step(h, dt);
        t = t + dt;
        ++n;
    }
    *t_inout = t;
    return n;
}
double orc_max_divb(void *p) {
    Handle *h = (Handle *)p;
    return h->counting ? h->c->find_divb() : h->d->find_divb();
}
/* unit hooks for the invariant tests */
void orc_recon_cell(int rec, const double *w, const double *v5, double *vm, double *vp) {
    double a, b;
    if (rec == CUMC_RECON_PPM) Sim<double>::ppmc(w, v5[0], v5[1], v5[2], v5[3], v5[4], a, b);
    else if (rec == CUMC_RECON_WENO) Sim<double>::weno(w, v5[0], v5[1], v5[2], v5[3], v5[4], a, b);
    else Sim<double>::tvd(rec, w, v5[1], v5[2], v5[3], a, b);
    *vm = a; *vp = b;
}
void orc_weights(int rec, const double *d5, double *w) {
    if (rec == CUMC_RECON_PPM) Sim<double>::ppm_interpolant(d5[0], d5[1], d5[2], d5[3], d5[4], w);
    else if (rec == CUMC_RECON_WENO) Sim<double>::weno_interpolant(d5[0], d5[1], d5[2], d5[3], d5[4], w);
    else { w[0] = (d5[2] + d5[3]) / d5[2]; w[1] = (d5[2] + d5[1]) / d5[2]; }
}
/* one face: BUILDSTATES + solver, states 1-based in arrays of 9 */
void orc_riemann_face(int dir, int rs, double gamma, const double *pl8, const double *pr8, double *fo8, double *fphys8) {
    cumc_config c;
    memset(&c, 0, sizeof c);
    Sim<double> s;
    s.cfg = c;
    s.cfg.riemann = rs;
    s.ggas = gamma;
    s.nx = s.ny = s.nz = 1; s.NX = s.NY = s.NZ = 7;
    size_t n3 = 343;
    s.primL.assign(8 * n3, 0.0); s.primR.assign(8 * n3, 0.0); s.uL.assign(8 * n3, 0.0); s.uR.assign(8 * n3, 0.0);
    s.fluxL.assign(8 * n3, 0.0); s.fluxR.assign(8 * n3, 0.0); s.flux.assign(8 * n3, 0.0);
    s.epsL.assign(n3, 0.0); s.epsR.assign(n3, 0.0); s.csL.assign(n3, 0.0); s.csR.assign(n3, 0.0);
    const int j = 1, k = 1, l = 1;
    for (int i = 1; i <= 8; ++i) { s.PL(i, j, k, l) = pl8[i - 1]; s.PR(i, j, k, l) = pr8[i - 1]; }
    size_t cc = s.c3(j, k, l);
    s.epsL[cc] = s.eos_eps(pl8[0], pl8[4]); s.epsR[cc] = s.eos_eps(pr8[0], pr8[4]);
    s.csL[cc] = s.eos_cs(pl8[4], pl8[0], s.epsL[cc]); s.csR[cc] = s.eos_cs(pr8[4], pr8[0], s.epsR[cc]);
    /* restrict the face loops to the single face (1,1,1) */
    s.nx = s.ny = s.nz = 1;
    s.buildstates(dir);
    s.riemann(dir);
    for (int i = 1; i <= 8; ++i) { fo8[i - 1] = s.FL(i, j, k, l); fphys8[i - 1] = s.FXL(i, j, k, l); }
}

/* ------------------------------------------------------------------ */
/* Learned smooth-face flag (no reference counterpart): the CPU checker */
/* of the GPU harvest, trainer and inference.  Features in float        */
/* arithmetic, labels from the FP64 WENO-Z of weno_module.f90:363-404.  */
/* ------------------------------------------------------------------ */
static void lrn_var_features(float a0, float a1, float a2, float a3, float a4, float *f4, float *r) {
    const float d0 = a1 - a0, d1 = a2 - a1, d2 = a3 - a2, d3 = a4 - a3;
    const float sum = ((std::fabs(d0) + std::fabs(d1)) + std::fabs(d2)) + std::fabs(d3);
    const float inv = 1.0f / (sum + 1.0e-30f);
    f4[0] = d0 * inv;
    f4[1] = d1 * inv;
    f4[2] = d2 * inv;
    f4[3] = d3 * inv;
    *r = sum * (1.0f / ((std::fabs(a2) + sum) + 1.0e-30f));
}

/* WENO-Z candidates P and indicators B of the right (p) and left (m) face */
static void lrn_parts(const double *w, double vm2, double vm1, double vc, double vp1, double vp2, double *Pp,
                      double *Bp, double *Pm, double *Bm) {
    double U01 = w[0] * vc + w[1] * vp1;
    double U12 = w[2] * vp1 + w[3] * vp2;
    double U10 = w[4] * vm1 + w[5] * vc;
    double U21 = w[6] * vm2 + w[7] * vm1;
    double U00 = vm1 + w[8] * (vm1 - vm2);
    double U11 = vp1 + w[9] * (vp1 - vp2);
    Pp[0] = (6.0 * vc - 1.0 * U10 - 2.0 * U00) / 3.0;
    Pp[1] = (-1.0 * U10 + 2.0 * vc + 2.0 * U01) / 3.0;
    Pp[2] = (2.0 * U01 + 2.0 * vp1 - 1.0 * U12) / 3.0;
    double t1 = 2.0 * U10 - 2.0 * U00, t2 = 4.0 * vc - 2.0 * U10 - 2.0 * U00;
    Bp[0] = r_weno_1 * (t1 * t1) + r_weno_2 * (t2 * t2);
    double t3 = 2.0 * U10 - 4.0 * vc + 2.0 * U01, t4 = -2.0 * U10 + 2.0 * U01;
    Bp[1] = r_weno_1 * (t3 * t3) + r_weno_2 * (t4 * t4);
    double t5 = 2.0 * U01 - 4.0 * vp1 + 2.0 * U12, t6 = -6.0 * U01 + 8.0 * vp1 - 2.0 * U12;
    Bp[2] = r_weno_1 * (t5 * t5) + r_weno_2 * (t6 * t6);
    Pm[0] = (6.0 * vc - 1.0 * U01 - 2.0 * U11) / 3.0;
    Pm[1] = (-1.0 * U01 + 2.0 * vc + 2.0 * U10) / 3.0;
    Pm[2] = (2.0 * U10 + 2.0 * vm1 - 1.0 * U21) / 3.0;
    t1 = 2.0 * U01 - 2.0 * U11; t2 = 4.0 * vc - 2.0 * U01 - 2.0 * U11;
    Bm[0] = r_weno_1 * (t1 * t1) + r_weno_2 * (t2 * t2);
    t3 = 2.0 * U01 - 4.0 * vc + 2.0 * U10; t4 = 2.0 * U01 - 2.0 * U10;
    Bm[1] = r_weno_1 * (t3 * t3) + r_weno_2 * (t4 * t4);
    t5 = 2.0 * U10 - 4.0 * vm1 + 2.0 * U21; t6 = 8.0 * vm1 - 6.0 * U10 - 2.0 * U21;
    Bm[2] = r_weno_1 * (t5 * t5) + r_weno_2 * (t6 * t6);
}

static void lrn_omega(const double *B, double *om) {
    const double tau5 = std::fabs(B[0] - B[2]);
    const double q1 = tau5 / (smallpara + B[0]), q2 = tau5 / (smallpara + B[1]), q3 = tau5 / (smallpara + B[2]);
    const double w1 = g_weno_1 * (1.0 + q1 * q1), w2 = g_weno_2 * (1.0 + q2 * q2), w3 = g_weno_3 * (1.0 + q3 * q3);
    const double sum = w1 + w2 + w3;
    om[0] = w1 / sum;
    om[1] = w2 / sum;
    om[2] = w3 / sum;
}

/* one sample: st = 7 stencils of 5 values (rho, v, p, the two transverse
 * cell fields), w = the cell's 10 WENO weights; row = 35 features, the
 * relative face-value change of the linear weights, the largest
 * nonlinear-weight deviation */
void orc_learn_sample(const double *st, const double *w, float *row) {
    const double g[3] = {g_weno_1, g_weno_2, g_weno_3};
    double change = 0.0, wdev = 0.0;
    for (int v = 0; v < 7; ++v) {
        const double *s5 = st + 5 * v;
        float f4[4], rv;
        lrn_var_features((float)s5[0], (float)s5[1], (float)s5[2], (float)s5[3], (float)s5[4], f4, &rv);
        for (int i = 0; i < 4; ++i) row[4 * v + i] = f4[i];
        row[28 + v] = rv;
        double Pp[3], Bp[3], Pm[3], Bm[3], om[3];
        lrn_parts(w, s5[0], s5[1], s5[2], s5[3], s5[4], Pp, Bp, Pm, Bm);
        lrn_omega(Bp, om);
        const double vp_z = om[0] * Pp[0] + om[1] * Pp[1] + om[2] * Pp[2];
        for (int q = 0; q < 3; ++q) wdev = std::fmax(wdev, std::fabs(om[q] - g[q]));
        lrn_omega(Bm, om);
        const double vm_z = om[0] * Pm[0] + om[1] * Pm[1] + om[2] * Pm[2];
        for (int q = 0; q < 3; ++q) wdev = std::fmax(wdev, std::fabs(om[q] - g[q]));
        const double vp_l = g[0] * Pp[0] + g[1] * Pp[1] + g[2] * Pp[2];
        const double vm_l = g[0] * Pm[0] + g[1] * Pm[1] + g[2] * Pm[2];
        const double den = std::fabs(s5[2]) + 1.0e-300;
        change = std::fmax(change, std::fmax(std::fabs(vp_l - vp_z), std::fabs(vm_l - vm_z)) / den);
    }
    row[35] = (float)change;
    row[36] = (float)wdev;
}

/* the flag network in FP64: parameters as the C-ABI (W1[32][48], b1,
 * W2[32][32], b2, w3, b3), samples of 37 floats, label change < delta.
 * Returns the mean binary cross-entropy; grad = its gradient. */
enum { L_H = 32, L_K = 48, L_NF = 35, L_ROW = 37, L_W1 = 0, L_B1 = 1536, L_W2 = 1568, L_B2 = 2592, L_W3 = 2624,
       L_B3 = 2656, L_NP = 2657 };
static double lrn_forward(const float *P, const float *x, double *h1, double *h2) {
    for (int o = 0; o < L_H; ++o) {
        double a = P[L_B1 + o];
        for (int i = 0; i < L_NF; ++i) a += (double)P[L_W1 + o * L_K + i] * (double)x[i];
        h1[o] = a > 0.0 ? a : 0.0;
    }
    for (int o = 0; o < L_H; ++o) {
        double a = P[L_B2 + o];
        for (int i = 0; i < L_H; ++i) a += (double)P[L_W2 + o * L_H + i] * h1[i];
        h2[o] = a > 0.0 ? a : 0.0;
    }
    double z = P[L_B3];
    for (int i = 0; i < L_H; ++i) z += (double)P[L_W3 + i] * h2[i];
    return z;
}

void orc_mlp_forward(const float *P, const float *X, int ld, long long n, double *z) {
    double h1[L_H], h2[L_H];
    for (long long s = 0; s < n; ++s) z[s] = lrn_forward(P, X + s * ld, h1, h2);
}

double orc_mlp_loss_grad(const float *P, const float *X, long long n, float delta, double *grad) {
    for (int p = 0; p < L_NP; ++p) grad[p] = 0.0;
    double loss = 0.0;
    double h1[L_H], h2[L_H], g1[L_H], g2[L_H];
    for (long long s = 0; s < n; ++s) {
        const float *x = X + s * L_ROW;
        const double y = x[L_NF] < delta ? 1.0 : 0.0;
        const double z = lrn_forward(P, x, h1, h2);
        loss += std::fmax(z, 0.0) - y * z + std::log1p(std::exp(-std::fabs(z)));
        const double dz = 1.0 / (1.0 + std::exp(-z)) - y;
        for (int i = 0; i < L_H; ++i) g2[i] = h2[i] > 0.0 ? dz * (double)P[L_W3 + i] : 0.0;
        for (int i = 0; i < L_H; ++i) {
            double a = 0.0;
            for (int o = 0; o < L_H; ++o) a += (double)P[L_W2 + o * L_H + i] * g2[o];
            g1[i] = h1[i] > 0.0 ? a : 0.0;
        }
        for (int o = 0; o < L_H; ++o) {
            for (int i = 0; i < L_NF; ++i) grad[L_W1 + o * L_K + i] += g1[o] * (double)x[i];
            grad[L_B1 + o] += g1[o];
            for (int i = 0; i < L_H; ++i) grad[L_W2 + o * L_H + i] += g2[o] * h1[i];
            grad[L_B2 + o] += g2[o];
            grad[L_W3 + o] += dz * h2[o];
        }
        grad[L_B3] += dz;
    }
    for (int p = 0; p < L_NP; ++p) grad[p] /= (double)n;
    return loss / (double)n;
}

/* Self-gravity potential of the collapsar model: GET_POISSON + POISSON_COEF
 * (model/collapsar/src/poisson.f90:6-64) and the red-black SOR loop of
 * CUSTOM_UPDATE (model/collapsar/src/custom.f90:511-620), restated with the
 * Fortran's loops and order: phi_old backup, abserror = 1e-50, red cells
 * ((-1)**(j+k+l) > 0) in l,k,j order, black cells, the error maximum, the
 * ghost layers, the exit test.  rho: interior, nx*ny*nz, j fastest; phi:
 * (nx+2)*(ny+2)*(nz+2), j fastest, j,k,l = 0..n+1, in/out.  A NaN error
 * (0/0 where phi stays zero) is kept as the maximum and fails the test.
 * Returns 1 when the error reached tol, 0 when max_iter ran out. */
int orc_poisson_solve(const cumc_config *cfg, const double *rho, double rho_atm, double omega, double tol,
                      int max_iter, double *phi, int *iters, double *err) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    const long long px = nx + 2, py = (long long)(nx + 2) * (ny + 2);
    // cell centres x(j) = (xF(j) + xF(j-1)) / 2 for j = 0..n+1 (getgrid.f90:55-63);
    // the face arrays start at index -3
    auto centre = [](const double *f, int j) { return (f[j + 3] + f[j + 2]) / 2.0; };
    std::vector<double> x(nx + 2), y(ny + 2), z(nz + 2);
    for (int j = 0; j <= nx + 1; ++j) x[j] = centre(cfg->xF, j);
    for (int k = 0; k <= ny + 1; ++k) y[k] = centre(cfg->yF, k);
    for (int l = 0; l <= nz + 1; ++l) z[l] = centre(cfg->zF, l);
    std::vector<double> ajp1(px), ajm1(px), bkp1(py), bkm1(py), clp1(py * (nz + 2)), clm1(py * (nz + 2)),
        epsc(py * (nz + 2));
    auto I3 = [&](int j, int k, int l) { return j + px * k + py * l; };
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j)
            for (int k = 1; k <= nz; ++k) {
                const double xm1 = x[i - 1], xc = x[i], xp1 = x[i + 1];
                const double ym1 = y[j - 1], yc = y[j], yp1 = y[j + 1];
                const double zm1 = z[k - 1], zc = z[k], zp1 = z[k + 1];
                epsc[I3(i, j, k)] = 2.0 * (xp1 + xm1 - 3.0 * xc) / xc / (xp1 - xc) / (xc - xm1) +
                                    (yp1 + ym1 - 2.0 * yc - 2.0 * std::tan(yc)) / (xc * xc) / std::tan(yc) /
                                        (yp1 - yc) / (yc - ym1) -
                                    2.0 / (xc * xc) / (std::sin(yc) * std::sin(yc)) / (zp1 - zc) / (zc - zm1);
                ajp1[i] = 2.0 * (2.0 * xc - xm1) / (xp1 - xm1) / (xp1 - xc) / xc;
                ajm1[i] = 2.0 * (2.0 * xc - xp1) / (xp1 - xm1) / (xc - xm1) / xc;
                bkp1[i + px * j] = (2.0 * std::tan(yc) + yc - ym1) / (xc * xc) / std::tan(yc) / (yp1 - yc) / (yp1 - ym1);
                bkm1[i + px * j] = (2.0 * std::tan(yc) + yc - yp1) / (xc * xc) / std::tan(yc) / (yp1 - ym1) / (yc - ym1);
                clp1[I3(i, j, k)] = 2.0 / (xc * xc) / (std::sin(yc) * std::sin(yc)) / (zp1 - zm1) / (zp1 - zc);
                clm1[I3(i, j, k)] = 2.0 / (xc * xc) / (std::sin(yc) * std::sin(yc)) / (zp1 - zm1) / (zc - zm1);
            }
    const double pi = 4.0 * std::atan(1.0);
    std::vector<double> phi_old(py * (nz + 2));
    auto sweep = [&](int parity) {
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    if (((j + k + l) & 1) != parity) continue;
                    const double r = rho[(j - 1) + (long long)nx * ((k - 1) + (long long)ny * (l - 1))];
                    const double diff = r - rho_atm;
                    const double factor = diff > 0.0 ? 1.0 : 0.0;
                    const double rho_in = factor * r;
                    const long long c = I3(j, k, l);
                    const double rhs = (4.0 * pi * rho_in -
                                        (ajp1[j] * phi[c + 1] + ajm1[j] * phi[c - 1] + bkp1[j + px * k] * phi[c + px] +
                                         bkm1[j + px * k] * phi[c - px] + clp1[c] * phi[c + py] + clm1[c] * phi[c - py])) /
                                       epsc[c];
                    phi[c] = (1.0 - omega) * phi[c] + omega * rhs;
                }
    };
    int n = 0, converged = 0;
    double abserror = 0.0;
    for (n = 1; n <= max_iter; ++n) {
        for (long long c = 0; c < py * (nz + 2); ++c) phi_old[c] = phi[c];
        abserror = 1.0e-50;
        sweep(0);  // red: (-1)**(j+k+l) > 0
        sweep(1);  // black
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k)
                for (int j = 1; j <= nx; ++j) {
                    const long long c = I3(j, k, l);
                    const double v = std::fabs((phi[c] - phi_old[c]) / phi_old[c]);
                    if (v != v || v > abserror) abserror = v;
                }
        for (int l = 1; l <= nz; ++l)
            for (int k = 1; k <= ny; ++k) {
                phi[I3(0, k, l)] = phi[I3(1, k, l)];
                phi[I3(nx + 1, k, l)] = -1.0;
            }
        for (int l = 1; l <= nz; ++l)
            for (int j = 1; j <= nx; ++j) {
                phi[I3(j, 0, l)] = phi[I3(j, 1, l)];
                phi[I3(j, ny + 1, l)] = phi[I3(j, ny, l)];
            }
        for (int k = 1; k <= ny; ++k)
            for (int j = 1; j <= nx; ++j) {
                phi[I3(j, k, 0)] = phi[I3(j, k, nz)];
                phi[I3(j, k, nz + 1)] = phi[I3(j, k, 1)];
            }
        if (abserror <= tol) {
            converged = 1;
            break;
        }
    }
    if (iters) *iters = converged ? n : max_iter;
    if (err) *err = abserror;
    return converged;
}

/* the collapsar model's black hole and potential (engine: cumc_collapsar_*,
 * cumc_poisson_*); phi: (nx+2)*(ny+2)*(nz+2), j fastest */
void orc_collapsar_set(void *p, double m_bh, double c_code) {
    Handle *h = (Handle *)p;
    auto set = [&](auto *s) {
        s->m_bh = m_bh;
        s->mbh_old = m_bh;
        s->c_code = c_code;
        s->r_sh = 2.0 * m_bh / (c_code * c_code);
    };
    if (h->counting) set(h->c); else set(h->d);
}
int orc_collapsar_get(void *p, double *m_bh, double *r_sh) {
    Handle *h = (Handle *)p;
    auto get = [&](auto *s) {
        *m_bh = s->m_bh;
        *r_sh = s->r_sh;
        return s->horizon_hit ? 1 : 0;
    };
    return h->counting ? get(h->c) : get(h->d);
}
void orc_set_phi(void *p, const double *phi) {
    Handle *h = (Handle *)p;
    auto set = [&](auto *s) { s->phi_.assign(phi, phi + (size_t)(s->nx + 2) * (s->ny + 2) * (s->nz + 2)); };
    if (h->counting) set(h->c); else set(h->d);
}

void orc_reset_counts(void) {
    for (int p = 0; p < N_PHASES; ++p) g_ops_ph[p] = OpCounts();
}
/* add, mul, div, sqrt, cmp summed over the phases (phase < 0) or of one
 * phase (0 the rest, 1 reconstruction, 2 BUILDSTATES + Riemann, 3 FINDDT) */
void orc_get_phase_counts(int phase, uint64_t *out5) {
    for (int i = 0; i < 5; ++i) out5[i] = 0;
    for (int p = 0; p < N_PHASES; ++p) {
        if (phase >= 0 && p != phase) continue;
        const OpCounts &c = g_ops_ph[p];
        out5[0] += c.add; out5[1] += c.mul; out5[2] += c.div; out5[3] += c.sqrt; out5[4] += c.cmp;
    }
}
void orc_get_counts(uint64_t *out5) { orc_get_phase_counts(-1, out5); }
/* OpenMP threads of the following calls (the reference hard-codes 4,
 * solver/mhd/main.f90:31; the baselines also run on every host core) */
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} /* extern "C" */
