// gauge_ops.cuh -- per-link operators of the constrained HMC path.
//
// Each function works on one link (x, mu) of one chain and is written once for
// float and double.  The staple and stout-derivative sums are reassociated so
// that sub-products shared between paths are formed once: the values are the
// reference sums (field-hmc.h:137-269, hep-lat/0311018 eq. 75 with
// field-multi.h:180-269), the matmul count per link drops from 85 to 51
// (Iwasaki staples, with double links) and from 66 to 37 (stout chain rule).
#pragma once

#include "lattice.cuh"

namespace magb {

// Sum of the forward-oriented staples of link (x, mu) with their action
// coefficients: A = sum_nu c0 (P_up + P_dn) + c1 (R1 + ... + R6), where the
// paths are those of get_staple_dagger (field-hmc.h:226-239) and
// get_rectangular_dagger (field-hmc.h:142-198).  The reference's
// get_extended_staple_dagger returns A^dag.
//
// The 1x2 rectangles use the double links W_nu(y) = U_nu(y) U_nu(y+nu) of the
// same field (k_double_link), so every path is two products:
//   R1 = U_nu(x) W_mu(x+nu) U_nu^dag(x+2mu) . U_mu^dag(x+mu)
//   R2 = U_nu^dag(x-nu) W_mu(x-nu) U_nu(x-nu+2mu) . U_mu^dag(x+mu)
//   R5 = U_mu^dag(x-mu) . U_nu(x-mu) W_mu(x-mu+nu) U_nu^dag(x+mu)
//   R6 = U_mu^dag(x-mu) . U_nu^dag(x-mu-nu) W_mu(x-mu-nu) U_nu(x-nu+mu)
//   R3 = W_nu(x) U_mu(x+2nu) W_nu^dag(x+mu)
//   R4 = W_nu^dag(x-2nu) U_mu(x-2nu) W_nu(x-2nu+mu)
// with the common factors U_mu^dag(x+mu), U_mu^dag(x-mu) applied once to the
// sums over nu.  Path products are special unitary: two rows are multiplied
// and the third reconstructed.
template <typename T, bool IWASAKI>
MAG_HD mat3<T> staple_sum(const LinkPlanes<T>& U, const LinkPlanes<T>& W, const ChainInfo& ci, const Site& st,
                          int mu) {
    mat3<T> A;
    set_zero(A);
    const T c0 = IWASAKI ? (T)ci.c0 : T(1);
    const T c1 = (T)ci.c1;
    if (IWASAKI) {
        // the +mu (R1, R2) and -mu (R5, R6) groups in one loop, one accumulator each
        mat3<T> accp, accm;
        set_zero(accp);
        set_zero(accm);
#pragma unroll 1
        for (int nu = 0; nu < 4; nu++) {
            if (nu == mu) continue;
            mat3<T> t = mul_2r(U.load_rows01(nu, st.g), W.load(mu, nb(ci, st, nu, 1)));
            add_to(accp, mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 2))));
            t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, nu, -1)), W.load(mu, nb(ci, st, nu, -1)));
            add_to(accp, mul_su3(t, U.load(nu, nb(ci, st, mu, 2, nu, -1))));
            t = mul_2r(U.load_rows01(nu, nb(ci, st, mu, -1)), W.load(mu, nb(ci, st, mu, -1, nu, 1)));
            add_to(accm, mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 1))));
            t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, mu, -1, nu, -1)), W.load(mu, nb(ci, st, mu, -1, nu, -1)));
            add_to(accm, mul_su3(t, U.load(nu, nb(ci, st, mu, 1, nu, -1))));
        }
        A = mul_nd(accp, U.load(mu, nb(ci, st, mu, 1)));
        mul_dn_acc(A, U.load(mu, nb(ci, st, mu, -1)), accm);
        A = scaled(A, c1);
    }
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        // P_up = U_nu(x) U_mu(x+nu) U_nu^dag(x+mu), P_dn = U_nu^dag(x-nu) U_mu(x-nu) U_nu(x-nu+mu)
        mat3<T> t = mul_2r(U.load_rows01(nu, st.g), U.load(mu, nb(ci, st, nu, 1)));
        axpy(A, c0, mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 1))));
        t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, nu, -1)), U.load(mu, nb(ci, st, nu, -1)));
        axpy(A, c0, mul_su3(t, U.load(nu, nb(ci, st, mu, 1, nu, -1))));
        if (IWASAKI) {
            t = mul_2r(W.load_rows01(nu, st.g), U.load(mu, nb(ci, st, nu, 2)));
            axpy(A, c1, mul_nd_su3(t, W.load(nu, nb(ci, st, mu, 1))));
            t = mul_dn_2r(W.load_cols01(nu, nb(ci, st, nu, -2)), U.load(mu, nb(ci, st, nu, -2)));
            axpy(A, c1, mul_su3(t, W.load(nu, nb(ci, st, mu, 1, nu, -2))));
        }
    }
    return A;
}

// The part of staple_sum that belongs to one direction nu != mu, in two
// halves for the direction-split kernels (one warp computes one half of one
// nu for 32 links):
//   ext : c1 [(R1 + R2) U_mu^dag(x+mu) + U_mu^dag(x-mu) (R5 + R6)]   (Iwasaki)
//   near: c0 (P_up + P_dn) + c1 (R3 + R4)
// The common factors U_mu^dag(x +- mu) multiply this plane's mu-extended
// rectangles alone (two more products per plane than staple_sum, which
// applies them once to the sums over nu).  Summed over both halves and the
// three nu it is A.
template <typename T, bool IWASAKI>
MAG_HD mat3<T> staple_part_ext(const LinkPlanes<T>& U, const LinkPlanes<T>& W, const ChainInfo& ci, const Site& st,
                               int mu, int nu) {
    mat3<T> A;
    if (!IWASAKI) {
        set_zero(A);
        return A;
    }
    mat3<T> t = mul_2r(U.load_rows01(nu, st.g), W.load(mu, nb(ci, st, nu, 1)));
    mat3<T> acc = mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 2)));
    t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, nu, -1)), W.load(mu, nb(ci, st, nu, -1)));
    add_to(acc, mul_su3(t, U.load(nu, nb(ci, st, mu, 2, nu, -1))));
    A = mul_nd(acc, U.load(mu, nb(ci, st, mu, 1)));
    t = mul_2r(U.load_rows01(nu, nb(ci, st, mu, -1)), W.load(mu, nb(ci, st, mu, -1, nu, 1)));
    acc = mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 1)));
    t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, mu, -1, nu, -1)), W.load(mu, nb(ci, st, mu, -1, nu, -1)));
    add_to(acc, mul_su3(t, U.load(nu, nb(ci, st, mu, 1, nu, -1))));
    mul_dn_acc(A, U.load(mu, nb(ci, st, mu, -1)), acc);
    return scaled(A, (T)ci.c1);
}
template <typename T, bool IWASAKI>
MAG_HD void staple_part_near_acc(mat3<T>& A, const LinkPlanes<T>& U, const LinkPlanes<T>& W, const ChainInfo& ci,
                                 const Site& st, int mu, int nu) {
    const T c0 = IWASAKI ? (T)ci.c0 : T(1);
    if (IWASAKI) {
        const T c1 = (T)ci.c1;
        mat3<T> t = mul_2r(W.load_rows01(nu, st.g), U.load(mu, nb(ci, st, nu, 2)));
        axpy(A, c1, mul_nd_su3(t, W.load(nu, nb(ci, st, mu, 1))));
        t = mul_dn_2r(W.load_cols01(nu, nb(ci, st, nu, -2)), U.load(mu, nb(ci, st, nu, -2)));
        axpy(A, c1, mul_su3(t, W.load(nu, nb(ci, st, mu, 1, nu, -2))));
    }
    mat3<T> t = mul_2r(U.load_rows01(nu, st.g), U.load(mu, nb(ci, st, nu, 1)));
    axpy(A, c0, mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 1))));
    t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, nu, -1)), U.load(mu, nb(ci, st, nu, -1)));
    axpy(A, c0, mul_su3(t, U.load(nu, nb(ci, st, mu, 1, nu, -1))));
}
// both halves of one nu
template <typename T, bool IWASAKI>
MAG_HD mat3<T> staple_part(const LinkPlanes<T>& U, const LinkPlanes<T>& W, const ChainInfo& ci, const Site& st,
                           int mu, int nu) {
    mat3<T> A = staple_part_ext<T, IWASAKI>(U, W, ci, st, mu, nu);
    staple_part_near_acc<T, IWASAKI>(A, U, W, ci, st, mu, nu);
    return A;
}

// Plaquette staple sum (the stout "stp", field-multi.h:34 with thin staples):
// sum_nu U_nu(x)U_mu(x+nu)U_nu^dag(x+mu) + U_nu^dag(x-nu)U_mu(x-nu)U_nu(x-nu+mu)
template <typename T>
MAG_HD mat3<T> plaq_staple_sum(const LinkPlanes<T>& U, const ChainInfo& ci, const Site& st, int mu) {
    mat3<T> A;
    set_zero(A);
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        mat3<T> t = mul_2r(U.load_rows01(nu, st.g), U.load(mu, nb(ci, st, nu, 1)));
        add_to(A, mul_nd_su3(t, U.load(nu, nb(ci, st, mu, 1))));
        t = mul_dn_2r(U.load_cols01(nu, nb(ci, st, nu, -1)), U.load(mu, nb(ci, st, nu, -1)));
        add_to(A, mul_su3(t, U.load(nu, nb(ci, st, mu, 1, nu, -1))));
    }
    return A;
}

// Chain rule of one stout level for link (x, mu), given Lambda on every link
// and Zp = Z' exp(iQ) at (x, mu).  Returns
//   Z = Z' e^{iQ} + i rho [stp^dag Lambda(x,mu) - sum_nu (six insertion terms)],
// the bracket T accumulated per staple, grouped around the shared products
//   D = U_nu(x+mu) U_mu^dag(x+nu),  E = D U_nu^dag(x) = P_up^dag,
//   G = U_mu^dag(x-nu) U_nu(x-nu),  U_nu^dag(x-nu+mu) G = P_dn^dag:
//   upper: D [U_nu^dag(x) (L_mu(x) - L_nu(x)) - L_mu(x+nu) U_nu^dag(x)] + L_nu(x+mu) E
//   lower: U_nu^dag(x-nu+mu) [G L_mu(x) - U_mu^dag(x-nu) (L_mu(x-nu) - L_nu(x-nu)) U_nu(x-nu)
//                             - L_nu(x-nu+mu) G]
// (stp^dag Lambda(x,mu) is distributed over the staples, so only T is live
// across the loop).
template <typename T>
MAG_HD mat3<T> stout_chain(const LinkPlanes<T>& U, const AlgPlanes<T>& Lam, const LinkPlanes<T>& Zp,
                           const ChainInfo& ci, const Site& st, int mu) {
    const herm8<T> lx = Lam.load(mu, st.g);  // Lambda(x, mu)
    mat3<T> t;
    set_zero(t);
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        {
            const mat3<T> unx = U.load(nu, st.g);
            // D and E are products of links: two rows and a reconstructed third
            const mat3<T> D = mul_nd_su3(U.load_rows01(nu, nb(ci, st, mu, 1)), U.load(mu, nb(ci, st, nu, 1)));
            const mat3<T> E = mul_nd_su3(D, unx);
            mul_hm_acc(t, Lam.load(nu, nb(ci, st, mu, 1)), E);
            herm8<T> dl = Lam.load(nu, st.g);
#pragma unroll
            for (int k = 0; k < 8; k++) dl.h[k] = lx.h[k] - dl.h[k];
            mat3<T> inner = mul_dn_mh(unx, dl);
            mul_hm_nd_sub(inner, Lam.load(mu, nb(ci, st, nu, 1)), unx);
            mul_acc(t, D, inner);
        }
        {
            const int gm = nb(ci, st, nu, -1);
            const mat3<T> umn = U.load(mu, gm);
            const mat3<T> unn = U.load(nu, gm);
            const mat3<T> G = mul_dn_su3(umn, unn);
            herm8<T> dl = Lam.load(mu, gm);
            const herm8<T> ln = Lam.load(nu, gm);
#pragma unroll
            for (int k = 0; k < 8; k++) dl.h[k] -= ln.h[k];
            mat3<T> inner = mul_mh(G, lx);
            mul_sub(inner, mul_dn_mh(umn, dl), unn);
            mul_hm_sub(inner, Lam.load(nu, nb(ci, st, mu, 1, nu, -1)), G);
            mul_dn_acc(t, U.load(nu, nb(ci, st, mu, 1, nu, -1)), inner);
        }
    }
    mat3<T> z = Zp.load(mu, st.g);  // Z' e^{iQ}
    add_to(z, times_i(t, (T)ci.rho));
    return z;
}

// The bracket of stout_chain for one direction nu != mu, in two halves for
// the direction-split kernels: the upper staple's terms (upper) and the lower
// staple's (lower_acc adds them to t).  Summed over both halves and the three
// nu and multiplied by i rho it is Z - Z' e^{iQ}.
template <typename T>
MAG_HD mat3<T> stout_chain_upper(const LinkPlanes<T>& U, const AlgPlanes<T>& Lam, const herm8<T>& lx,
                                 const ChainInfo& ci, const Site& st, int mu, int nu) {
    const mat3<T> unx = U.load(nu, st.g);
    const mat3<T> D = mul_nd_su3(U.load_rows01(nu, nb(ci, st, mu, 1)), U.load(mu, nb(ci, st, nu, 1)));
    const mat3<T> E = mul_nd_su3(D, unx);
    mat3<T> t = mul_hm(Lam.load(nu, nb(ci, st, mu, 1)), E);
    herm8<T> dl = Lam.load(nu, st.g);
#pragma unroll
    for (int k = 0; k < 8; k++) dl.h[k] = lx.h[k] - dl.h[k];
    mat3<T> inner = mul_dn_mh(unx, dl);
    mul_hm_nd_sub(inner, Lam.load(mu, nb(ci, st, nu, 1)), unx);
    mul_acc(t, D, inner);
    return t;
}
template <typename T>
MAG_HD void stout_chain_lower_acc(mat3<T>& t, const LinkPlanes<T>& U, const AlgPlanes<T>& Lam, const herm8<T>& lx,
                                  const ChainInfo& ci, const Site& st, int mu, int nu) {
    const int gm = nb(ci, st, nu, -1);
    const mat3<T> umn = U.load(mu, gm);
    const mat3<T> unn = U.load(nu, gm);
    const mat3<T> G = mul_dn_su3(umn, unn);
    herm8<T> dl = Lam.load(mu, gm);
    const herm8<T> ln = Lam.load(nu, gm);
#pragma unroll
    for (int k = 0; k < 8; k++) dl.h[k] -= ln.h[k];
    mat3<T> inner = mul_mh(G, lx);
    mul_sub(inner, mul_dn_mh(umn, dl), unn);
    mul_hm_sub(inner, Lam.load(nu, nb(ci, st, mu, 1, nu, -1)), G);
    mul_dn_acc(t, U.load(nu, nb(ci, st, mu, 1, nu, -1)), inner);
}

// Lambda of compute_Lambda (field-multi.h:180-269) and Z' exp(iQ) for one link.
template <typename T>
MAG_HD void stout_lambda(const herm8<T>& q, const mat3<T>& Z, const mat3<T>& Ul, herm8<T>& lam, mat3<T>& zp) {
    const mat3<T> Q = expand(q);
    const mat3<T> QQ = mul_hm(q, Q);
    cplx<T> f0, f1, f2, b10, b11, b12, b20, b21, b22;
    bool nontrivial;
    if constexpr (sizeof(T) == 4) {
        ch_coef_f c;
        nontrivial = ch_for<T, true>(Q, QQ, c);  // FP32: power series (see su3.cuh)
        f0 = mk(c.f0r, c.f0i); f1 = mk(c.f1r, c.f1i); f2 = mk(c.f2r, c.f2i);
        b10 = mk(c.b10r, c.b10i); b11 = mk(c.b11r, c.b11i); b12 = mk(c.b12r, c.b12i);
        b20 = mk(c.b20r, c.b20i); b21 = mk(c.b21r, c.b21i); b22 = mk(c.b22r, c.b22i);
    } else {
        double c0, c1;
        ch_invariants(Q, QQ, c0, c1);
        const ch_coef c = ch_coefficients<true>(c0, c1);  // FP64: the reference's closed form
        nontrivial = !c.trivial;
        f0 = mk<T>(c.f0r, c.f0i); f1 = mk<T>(c.f1r, c.f1i); f2 = mk<T>(c.f2r, c.f2i);
        b10 = mk<T>(c.b10r, c.b10i); b11 = mk<T>(c.b11r, c.b11i); b12 = mk<T>(c.b12r, c.b12i);
        b20 = mk<T>(c.b20r, c.b20i); b21 = mk<T>(c.b21r, c.b21i); b22 = mk<T>(c.b22r, c.b22i);
    }
    if (!nontrivial) {
        // c1 = 0: exp(iQ) = 1 and Lambda = 0 (field-multi.h:190)
        zp = Z;
        lam = herm_zero<T>();
        return;
    }
    // exp(iQ) = f0 + f1 Q + f2 Q^2 and Z' exp(iQ)
    mat3<T> eq;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cplx<T> e = cmul<false, false>(f1, Q.e[i][j]);
            cmac<false, false, false>(e, f2, QQ.e[i][j]);
            eq.e[i][j] = e;
        }
#pragma unroll
    for (int i = 0; i < 3; i++) eq.e[i][i] = eq.e[i][i] + f0;
    zp = mul(Z, eq);
    const mat3<T> W = mul(Ul, Z);  // U Sigma'
    // Tr(Sigma' B U) = Tr(B W) with B = b0 + b1 Q + b2 Q^2
    const cplx<T> trW = mk<T>(W.e[0][0].re + W.e[1][1].re + W.e[2][2].re, W.e[0][0].im + W.e[1][1].im + W.e[2][2].im);
    const cplx<T> trQW = tr_mul(Q, W), trQQW = tr_mul(QQ, W);
    cplx<T> t1 = cmul<false, false>(b10, trW);
    cmac<false, false, false>(t1, b11, trQW);
    cmac<false, false, false>(t1, b12, trQQW);
    cplx<T> t2 = cmul<false, false>(b20, trW);
    cmac<false, false, false>(t2, b21, trQW);
    cmac<false, false, false>(t2, b22, trQQW);
    // Gamma = t1 Q + t2 Q^2 + f1 W + f2 (Q W + W Q)
    mat3<T> QW = mul_hm(q, W);
    mul_mh_acc(QW, W, q);
    mat3<T> G;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            cplx<T> g = cmul<false, false>(t1, Q.e[i][j]);
            cmac<false, false, false>(g, t2, QQ.e[i][j]);
            cmac<false, false, false>(g, f1, W.e[i][j]);
            cmac<false, false, false>(g, f2, QW.e[i][j]);
            G.e[i][j] = g;
        }
    lam = herm_traceless(G);
}

// Link update of evolve_gauge_field (field-hmc.h:442-482) with X = momentum or
// force and step eps:  0: e^{i eps X(x)} U;  1: e^{i eps X(x-mu)} U e^{-i eps X(x)};
// 10: U e^{-i eps X(x)};  100: e^{i eps X(x-mu)} U.  One exponential per link
// (two for the interior links of a segment, case 1, which only mag >= 3 has),
// evaluated at one call site in a loop so that it is inlined once.
template <typename TU, typename TX>
MAG_HD mat3<TU> evolve_link(const mat3<TU>& u, const AlgPlanes<TX>& X, double eps, int ccase, int g, int gm, int mu) {
    mat3<TU> r = u;
    const int nexp = ccase == 1 ? 2 : 1;
#pragma unroll 1
    for (int k = 0; k < nexp; k++) {
        // left factor e^{i eps X(y)} (cases 0, 100, and 1 first) or right factor e^{-i eps X(x)} (10, 1 second)
        const bool right = ccase == 10 || k == 1;
        const int y = (ccase == 100 || (ccase == 1 && k == 0)) ? gm : g;
        const herm8<TX> xl = X.load(mu, y);
        const TU s = (TU)(right ? -eps : eps);
        herm8<TU> q;
#pragma unroll
        for (int j = 0; j < 8; j++) q.h[j] = (TU)xl.h[j] * s;
        const mat3<TU> e = expiQ(q);
        r = right ? mul(r, e) : mul(e, r);
    }
    return r;
}

// ReTr of the six plaquettes at x (field-matrix.h:202-221 get_plaq)
template <typename T>
MAG_HD double site_plaquette(const LinkPlanes<T>& U, const ChainInfo& ci, const Site& st) {
    double s = 0.0;
#pragma unroll 1
    for (int mu = 1; mu < 4; mu++) {
        const mat3<T> umu = U.load(mu, st.g);
#pragma unroll 1
        for (int nu = 0; nu < mu; nu++) {
            const mat3<T> m = mul(umu, U.load(nu, nb(ci, st, mu, 1)));
            const mat3<T> n = mul(U.load(nu, st.g), U.load(mu, nb(ci, st, nu, 1)));
            s += (double)retr(mul_nd(m, n));
        }
    }
    return s;
}

// ReTr of the twelve 1x2 rectangles at x (field-matrix.h:249-297 get_rectangular)
template <typename T>
MAG_HD double site_rectangle(const LinkPlanes<T>& U, const ChainInfo& ci, const Site& st) {
    double s = 0.0;
#pragma unroll 1
    for (int mu = 1; mu < 4; mu++) {
        const mat3<T> umu = U.load(mu, st.g);
        const int gm = nb(ci, st, mu, 1);
#pragma unroll 1
        for (int nu = 0; nu < mu; nu++) {
            const mat3<T> unu = U.load(nu, st.g);
            const int gn = nb(ci, st, nu, 1);
            const int gmn = nb(ci, st, mu, 1, nu, 1);
            // (U_mu(x) U_nu(x+mu) U_nu(x+mu+nu))^dag vs U_nu(x) U_nu(x+nu) U_mu(x+2nu)
            mat3<T> a = mul(mul(umu, U.load(nu, gm)), U.load(nu, gmn));
            mat3<T> b = mul(mul(unu, U.load(nu, gn)), U.load(mu, nb(ci, st, nu, 2)));
            s += (double)retr(mul_nd(b, a));
            // (U_mu(x) U_mu(x+mu) U_nu(x+2mu))^dag vs U_nu(x) U_mu(x+nu) U_mu(x+mu+nu)
            a = mul(mul(umu, U.load(mu, gm)), U.load(nu, nb(ci, st, mu, 2)));
            b = mul(mul(unu, U.load(mu, gn)), U.load(mu, gmn));
            s += (double)retr(mul_nd(b, a));
        }
    }
    return s;
}

}  // namespace magb
