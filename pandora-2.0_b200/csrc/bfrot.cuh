// bfrot.cuh -- homogeneous shear in Rogallo (moving-frame) coordinates, the
// "Bardino/Ferziger rotational" (BF-rot, NS_DEFORMED = 1) formulation.
//
// Transformation tensors as set by g_DomainCalc (src/pg_domain.f90:187-214):
// binv = diag(B110, B220, B330) plus binv(1,3); bmat = diag(1/B110, 1/B220,
// 1/B330) plus bmat(1,3); amat(1,3) = S.  Entries that exist: the diagonal and
// (1,3) (bvalexist), and amat(1,3) (avalexist).  bmat(1,3), binv(1,3) follow the
// closed form of g_RK3UpdateB (src/pg_rk3.f90:280-385) and live in the Clock.
#pragma once
#include "pandora_internal.cuh"

namespace pd {

// The frame's tensors in real type R: FP64 as computed, or rounded once to FP32 for
// the pointwise products of the FP32-mixed form (bf_as).
template <class R> struct BFT {
    R bm[3][3];
    R bi[3][3];
    R a13;     // amat(1,3) = F_DEFORM_S
};
using BF = BFT<double>;

__host__ __device__ __forceinline__ constexpr bool bex(int a, int b) { return a == b || (a == 0 && b == 2); }

__device__ __forceinline__ BF make_bf(const Geo& g, const Clock* ck) {
    BF f;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) { f.bm[a][b] = 0.0; f.bi[a][b] = 0.0; }
    f.bm[0][0] = g.bdiag[0]; f.bm[1][1] = g.bdiag[1]; f.bm[2][2] = g.bdiag[2];
    f.bi[0][0] = g.bidiag[0]; f.bi[1][1] = g.bidiag[1]; f.bi[2][2] = g.bidiag[2];
    f.bm[0][2] = ck->b13;
    f.bi[0][2] = ck->bi13;
    f.a13 = g.shear_s;
    return f;
}

template <class R> __device__ __forceinline__ BFT<R> bf_as(const BF& f) {
    BFT<R> r;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) { r.bm[a][b] = (R)f.bm[a][b]; r.bi[a][b] = (R)f.bi[a][b]; }
    r.a13 = (R)f.a13;
    return r;
}

// f_RK3VorticityBFRot (src/pf_rk3.f90:3786-3843), summed over the three velocity
// components: w = sum_n omega(u_n).  Structurally w[0] has no term in u[0] and
// w[1] none in u[1] (bex), so a caller that needs only w[0] or w[1] may pass zero
// for that component.
// ONLY >= 0: only component ONLY of w is formed (the others are left zero).
template <int ONLY = -1, class R, class C>
__device__ __forceinline__ void vort_bf(const BFT<R>& f, const C* u, const R* k, C* w) {
    w[0].x = R(0); w[0].y = R(0); w[1] = w[0]; w[2] = w[0];
#pragma unroll
    for (int n = 0; n < 3; n++) {
        const C un = u[n];
#pragma unroll
        for (int m = 0; m < 3; m++) {
            if (bex(m, 0)) {
                if ((ONLY < 0 || ONLY == 1) && bex(2, n)) { const R c = f.bm[m][0] * f.bi[2][n] * k[m]; w[1].y -= c * un.x; w[1].x += c * un.y; }
                if ((ONLY < 0 || ONLY == 2) && bex(1, n)) { const R c = f.bm[m][0] * f.bi[1][n] * k[m]; w[2].y += c * un.x; w[2].x -= c * un.y; }
            }
            if (bex(m, 1)) {
                if ((ONLY < 0 || ONLY == 0) && bex(2, n)) { const R c = f.bm[m][1] * f.bi[2][n] * k[m]; w[0].y += c * un.x; w[0].x -= c * un.y; }
                if ((ONLY < 0 || ONLY == 2) && bex(0, n)) { const R c = f.bm[m][1] * f.bi[0][n] * k[m]; w[2].y -= c * un.x; w[2].x += c * un.y; }
            }
            if (bex(m, 2)) {
                if ((ONLY < 0 || ONLY == 0) && bex(1, n)) { const R c = f.bm[m][2] * f.bi[1][n] * k[m]; w[0].y -= c * un.x; w[0].x += c * un.y; }
                if ((ONLY < 0 || ONLY == 1) && bex(0, n)) { const R c = f.bm[m][2] * f.bi[0][n] * k[m]; w[1].y += c * un.x; w[1].x -= c * un.y; }
            }
        }
    }
}

// R-rot form (NS_DEFORMED = NS_R_ROT): the velocity components are laboratory ones on
// the sheared wavenumber grid.  f_RK3DerivativeRRot (src/pf_rk3.f90:3749-3780):
// d/dx_j = i sum_m bmat(m,j) k_m over every m; the vorticity w = D x u assembled per
// velocity component as the reference does (src/pf_rk3.f90:416-421, 470-475, 585-590).
template <class R, class C>
__device__ __forceinline__ C deriv_rrot(const BFT<R>& f, C u, const R* k, int j) {
    C d;
    d.x = R(0); d.y = R(0);
#pragma unroll
    for (int m = 0; m < 3; m++) {
        d.y = d.y + (f.bm[m][j] * k[m] * u.x);
        d.x = d.x - (f.bm[m][j] * k[m] * u.y);
    }
    return d;
}
// ONLY >= 0: only component ONLY of w is formed, from its two derivatives (the others
// are left zero); the same operations in the same order as for all three.
template <int ONLY = -1, class R, class C>
__device__ __forceinline__ void vort_rrot(const BFT<R>& f, const C* u, const R* k, C* w) {
    constexpr bool A0 = ONLY < 0 || ONLY == 0, A1 = ONLY < 0 || ONLY == 1, A2 = ONLY < 0 || ONLY == 2;
    w[0].x = R(0); w[0].y = R(0); w[1] = w[0]; w[2] = w[0];
    if constexpr (A1) w[1] = deriv_rrot(f, u[0], k, 2);
    if constexpr (A2) {
        const C dudy = deriv_rrot(f, u[0], k, 1);
        w[2].x = -dudy.x; w[2].y = -dudy.y;
    }
    if constexpr (A0) {
        const C dvdz = deriv_rrot(f, u[1], k, 2);
        w[0].x = w[0].x - dvdz.x; w[0].y = w[0].y - dvdz.y;
    }
    if constexpr (A2) {
        const C dvdx = deriv_rrot(f, u[1], k, 0);
        w[2].x = w[2].x + dvdx.x; w[2].y = w[2].y + dvdx.y;
    }
    if constexpr (A0) {
        const C dwdy = deriv_rrot(f, u[2], k, 1);
        w[0].x = w[0].x + dwdy.x; w[0].y = w[0].y + dwdy.y;
    }
    if constexpr (A1) {
        const C dwdx = deriv_rrot(f, u[2], k, 0);
        w[1].x = w[1].x - dwdx.x; w[1].y = w[1].y - dwdx.y;
    }
}

// f_RK3FormFRRot for F_SHEAR_DNS (src/pf_rk3.f90:2680-2856): viscous (f_RK3RRotViscous)
// - NL + pressure (f_RK3RRotPressure) - source A u (f_RK3RRotSource); the nonlinear
// term enters as computed (the isotropic product of the R-rot vorticity).
__device__ __forceinline__ void rhs_rrot(const BF& f, double nu, const double* k, const double2* u,
                                         const double2* nl, double2* tot) {
    double p1[3] = {0.0, 0.0, 0.0}, p4 = 0.0;
    double2 p2 = make_double2(0.0, 0.0), p3 = p2;
#pragma unroll
    for (int m = 0; m < 3; m++)
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (!bex(m, r)) continue;
            p2.x = p2.x + (k[m] * f.bm[m][r] * nl[r].x);
            p2.y = p2.y + (k[m] * f.bm[m][r] * nl[r].y);
            if (r == 0) {   // amat(r, q) exists only for (r, q) = (1, 3)
                p3.x = p3.x + (k[m] * f.bm[m][r] * f.a13 * u[2].x);
                p3.y = p3.y + (k[m] * f.bm[m][r] * f.a13 * u[2].y);
            }
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (bex(q, r)) p4 = p4 + (k[m] * f.bm[m][r] * k[q] * f.bm[q][r]);
        }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int pp = 0; pp < 3; pp++)
            if (bex(pp, a)) p1[a] = p1[a] + k[pp] * f.bm[pp][a];
    double2 visc[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
#pragma unroll
    for (int l = 0; l < 3; l++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
            if (!bex(l, jj)) continue;
#pragma unroll
            for (int n = 0; n < 3; n++) {
                if (!bex(n, jj)) continue;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    visc[a].x = visc[a].x - nu * f.bm[l][jj] * f.bm[n][jj] * k[l] * k[n] * u[a].x;
                    visc[a].y = visc[a].y - nu * f.bm[l][jj] * f.bm[n][jj] * k[l] * k[n] * u[a].y;
                }
            }
        }
    // one reciprocal for the three components (FP64 division is a long instruction
    // sequence; the product differs from the quotient by at most an ulp)
    const double ip4 = (p4 > 0.0) ? 1.0 / p4 : 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double2 pr = (p4 > 0.0) ? make_double2((p1[a] * ip4) * (p2.x + p3.x), (p1[a] * ip4) * (p2.y + p3.y))
                                      : make_double2(0.0, 0.0);
        const double2 hom = (a == 0) ? make_double2(f.a13 * u[2].x, f.a13 * u[2].y) : make_double2(0.0, 0.0);
        tot[a] = make_double2(visc[a].x - nl[a].x + pr.x + 0.0 - hom.x, visc[a].y - nl[a].y + pr.y + 0.0 - hom.y);
    }
}

// f_RK3ContinuityFixRRot (src/pf_rk3.f90:3620-3693): project the moving components
// bmat u on the (unsheared) wave vector, back with binv.
__device__ __forceinline__ void contfix_rrot(const BF& f, const double* k, double kmag2, double2* u) {
    double2 um[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
            if (bex(a, b)) { um[a].x = um[a].x + (f.bm[a][b] * u[b].x); um[a].y = um[a].y + (f.bm[a][b] * u[b].y); }
    const double2 kdu = make_double2(k[0] * um[0].x + k[1] * um[1].x + k[2] * um[2].x,
                                     k[0] * um[0].y + k[1] * um[1].y + k[2] * um[2].y);
    const double ik2 = 1.0 / kmag2;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        um[a].x = um[a].x - (k[a] * kdu.x * ik2);
        um[a].y = um[a].y - (k[a] * kdu.y * ik2);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
        u[a] = make_double2(0.0, 0.0);
#pragma unroll
        for (int b = 0; b < 3; b++)
            if (bex(a, b)) { u[a].x = u[a].x + (f.bi[a][b] * um[b].x); u[a].y = u[a].y + (f.bi[a][b] * um[b].y); }
    }
}

// f_ArraysDealiasSpherical / f_ArraysLESCutoff (src/pf_arrays.f90:1865-1987): a mode
// whose laboratory-frame wave vector k_lab(n) = sum_m bmat(m,n) k(m) is longer than
// g.dealias_cut is dropped.  Unfused, correctly rounded products and sums in the
// reference's order, so that the decision at the cutoff is the reference's.
__device__ __forceinline__ bool dealias_drop(const Geo& g, const BF& f, double k1, double k2, double k3) {
    const double kv[3] = {k1, k2, k3};
    double kl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < 3; m++)
#pragma unroll
        for (int n = 0; n < 3; n++)
            if (bex(m, n)) kl[n] = __dadd_rn(kl[n], __dmul_rn(f.bm[m][n], kv[m]));
    const double km = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(kl[0], kl[0]), __dmul_rn(kl[1], kl[1])), __dmul_rn(kl[2], kl[2])));
    return km > g.dealias_cut;
}

// f_RK3ComputeNonlinearBFRot (src/pf_rk3.f90:1634-1711), pointwise in physical space.
template <class R>
__device__ __forceinline__ void nl_bf(const BFT<R>& f, const R* u, const R* om, R* nl) {
    // omega x (binv u): the laboratory velocity first (binv has the diagonal and (1,3)),
    // then the cross product -- the reference's sum over the entries of binv, regrouped
    const R v0 = f.bi[0][0] * u[0] + f.bi[0][2] * u[2], v1 = f.bi[1][1] * u[1], v2 = f.bi[2][2] * u[2];
    nl[0] = om[1] * v2 - om[2] * v1;
    nl[1] = om[2] * v0 - om[0] * v2;
    nl[2] = om[0] * v1 - om[1] * v0;
}

// Right-hand side of f_RK3FormFBFRot for F_SHEAR_DNS (src/pf_rk3.f90:2494-2673):
// viscous (2903-2937) - bmat NL (2864-2895) + pressure (2986-3070) - source
// (3167-3209).  amat has the single entry (1,3).
__device__ __forceinline__ void rhs_bf(const BF& f, double nu, const double* k, const double2* u,
                                       const double2* nlr, double2* tot) {
    double2 nl[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        nl[a] = make_double2(0.0, 0.0);
#pragma unroll
        for (int b = 0; b < 3; b++)
            if (bex(a, b)) { nl[a].x += f.bm[a][b] * nlr[b].x; nl[a].y += f.bm[a][b] * nlr[b].y; }
    }
    // pressure
    double p1[3] = {0.0, 0.0, 0.0}, p4 = 0.0;
    double2 p2 = make_double2(0.0, 0.0), p3 = p2;
#pragma unroll
    for (int m = 0; m < 3; m++) {
        p2.x += k[m] * nl[m].x; p2.y += k[m] * nl[m].y;
#pragma unroll
        for (int r = 0; r < 3; r++) {
            if (!bex(m, r)) continue;
            if (r == 0) {   // amat(r, s) exists only for (r, s) = (1, 3)
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    if (!bex(2, q)) continue;
                    const double c = k[m] * f.bm[m][r] * f.a13 * f.bi[2][q];
                    p3.x += 2.0 * (c * u[q].x); p3.y += 2.0 * (c * u[q].y);
                }
            }
#pragma unroll
            for (int q = 0; q < 3; q++)
                if (bex(q, r)) p4 += k[m] * f.bm[m][r] * f.bm[q][r] * k[q];
        }
    }
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int pp = 0; pp < 3; pp++)
            if (bex(a, pp))
#pragma unroll
                for (int b = 0; b < 3; b++)
                    if (bex(b, pp)) p1[a] += f.bm[a][pp] * f.bm[b][pp] * k[b];
    // homogeneous source
    double2 hom[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        hom[a] = make_double2(0.0, 0.0);
        if (bex(a, 0)) {   // r = 1 is the only row of amat
#pragma unroll
            for (int q = 0; q < 3; q++) {
                if (!bex(2, q)) continue;
                const double c = f.bm[a][0] * f.a13 * f.bi[2][q];
                hom[a].x += 2.0 * (c * u[q].x); hom[a].y += 2.0 * (c * u[q].y);
            }
        }
    }
    // viscous
    double vc = 0.0;
#pragma unroll
    for (int l = 0; l < 3; l++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
            if (!bex(l, jj)) continue;
#pragma unroll
            for (int n = 0; n < 3; n++)
                if (bex(n, jj)) vc += nu * f.bm[l][jj] * f.bm[n][jj] * k[l] * k[n];
        }
    // one reciprocal for the three components (FP64 division is a long instruction
    // sequence; the product differs from the quotient by at most an ulp)
    const double ip4 = (p4 > 0.0) ? 1.0 / p4 : 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double2 pr = (p4 > 0.0) ? make_double2((p1[a] * ip4) * (p2.x + p3.x), (p1[a] * ip4) * (p2.y + p3.y))
                                      : make_double2(0.0, 0.0);
        tot[a] = make_double2(-vc * u[a].x - nl[a].x + pr.x - hom[a].x, -vc * u[a].y - nl[a].y + pr.y - hom[a].y);
    }
}

// g_RK3UpdateB (src/pg_rk3.f90:280-385): closed-form bmat(1,3), binv(1,3) of a
// shear flow at stage-end time `simtime` of step `tstep`.
__host__ __device__ __forceinline__ void update_b(const Geo& g, int tstep, double simtime, double& b13,
                                                  double& bi13) {
    double localtime = simtime;
    if (g.rk3_decide && tstep > g.b110 * g.remesh_t) {
        const int a = tstep - (g.b110 * g.remesh_t) - 1;
        const int b = 2 * (g.b110 * g.remesh_t);
        const int lt = a / b;
        localtime = simtime - ((double)(lt + 1) / g.shear_s * (double)g.b110);
    }
    b13 = -g.bdiag[0] * g.shear_s * localtime;
    bi13 = g.shear_s * localtime / g.bdiag[2];
}

__host__ __device__ __forceinline__ bool remesh_due(const Geo& g, int tstep) {
    if (!g.shear || !g.rk3_decide) return false;
    const int a = tstep - (g.b110 * g.remesh_t) - 1;
    const int b = 2 * g.b110 * g.remesh_t;
    return (a % b) == 0;
}

}  // namespace pd
