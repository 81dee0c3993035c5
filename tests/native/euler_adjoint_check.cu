// Host-side check of the Euler reverse-mode adjoints (PhysEuler::volume_adj / inner_adj)
// against forward-mode DualN differentiation of the primal volume() / inner() functors on
// random states covering all HLLC branches (upwind side, star region, pStar clamp, shock
// factors). Exit status 0 if every gradient agrees to 1e-11 relative; prints the worst case.
#include <cmath>
#include <cstdio>
#include <random>

#include "../../bosss_b200/csrc/dg_physics.cuh"

using namespace bosss;
constexpr int D = 3, NV = 5;
using E3 = PhysEuler<D>;

static void state(std::mt19937_64& g, double un_scale, double* U) {
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    double rho = 1.0 + 0.5 * u(g), p = 1.0 + 0.6 * u(g);
    double v[D];
    for (int d = 0; d < D; ++d) v[d] = un_scale * u(g);
    U[0] = rho;
    double ke = 0.0;
    for (int d = 0; d < D; ++d) {
        U[d + 1] = rho * v[d];
        ke += v[d] * v[d];
    }
    // p = (gamma-1)(E - 0.5 gMs rho |v|^2) with gMs = 1 below
    U[D + 1] = p / 0.4 + 0.5 * rho * ke;
}

int main() {
    PhysParams ph{};
    ph.gamma = 1.4;
    ph.mach = 1.0 / std::sqrt(1.4);
    ph.ims = 1.0 / (ph.gamma * ph.mach * ph.mach);
    ph.imach = 1.0 / ph.mach;
    std::mt19937_64 g(1234);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    double worst = 0.0;
    int branches[2][2] = {{0, 0}, {0, 0}}, clamps = 0, shocks = 0;
    for (int it = 0; it < 20000; ++it) {
        const double scale = (it % 4 == 0) ? 3.0 : (it % 4 == 1 ? 1.2 : 0.4);
        double UA[NV], UB[NV], n[D], fb[NV], Gw[NV][D];
        state(g, scale, UA);
        state(g, scale, UB);
        if (it % 3 == 0) {
            for (int d = 0; d < D; ++d) n[d] = 0.0;
            n[it % D] = (it % 2) ? 1.0 : -1.0;
        } else {
            double nn = 0.0;
            for (int d = 0; d < D; ++d) {
                n[d] = u(g);
                nn += n[d] * n[d];
            }
            for (int d = 0; d < D; ++d) n[d] /= std::sqrt(nn);
        }
        for (int e = 0; e < NV; ++e) {
            fb[e] = u(g);
            for (int d = 0; d < D; ++d) Gw[e][d] = u(g);
        }
        // ---- volume
        {
            using T = DualN<NV>;
            T U[NV], Gr[NV][D], fV[NV], fG[NV][D];
            for (int i = 0; i < NV; ++i) {
                U[i] = T(UA[i]);
                U[i].d[i] = 1.0;
                for (int d = 0; d < D; ++d) Gr[i][d] = T(0.0);
            }
            for (int e = 0; e < NV; ++e) {
                fV[e] = T(0.0);
                for (int d = 0; d < D; ++d) fG[e][d] = T(0.0);
            }
            E3::volume(ph, U, Gr, n, fV, fG);
            T phi(0.0);
            for (int e = 0; e < NV; ++e)
                for (int d = 0; d < D; ++d) phi += fG[e][d] * Gw[e][d];
            double Ub[NV];
            E3::volume_adj(ph, UA, Gw, Ub);
            double mx = 0.0, df = 0.0;
            for (int i = 0; i < NV; ++i) {
                mx = std::fmax(mx, std::fabs(phi.d[i]));
                df = std::fmax(df, std::fabs(phi.d[i] - Ub[i]));
            }
            worst = std::fmax(worst, df / mx);
        }
        // ---- HLLC face, both sides
        for (int side = 0; side < 2; ++side) {
            using T = DualN<NV>;
            T A[NV], B[NV], GA[NV][D], GB[NV][D], gA[NV], gB[NV], GAv[NV][D], GBv[NV][D];
            for (int i = 0; i < NV; ++i) {
                A[i] = T(UA[i]);
                B[i] = T(UB[i]);
                (side == 0 ? A[i] : B[i]).d[i] = 1.0;
                gA[i] = gB[i] = T(0.0);
                for (int d = 0; d < D; ++d) GA[i][d] = GB[i][d] = GAv[i][d] = GBv[i][d] = T(0.0);
            }
            E3::inner(ph, 0.0, A, GA, B, GB, n, n, gA, GAv, gB, GBv);
            // gA = +f, gB = -f: sum_e gA_e w_e with w = fb gives sum f fb
            T phi(0.0);
            for (int e = 0; e < NV; ++e) phi += gA[e] * fb[e];
            double UAb[NV], UBb[NV];
            E3::inner_adj(ph, UA, UB, n, fb, UAb, UBb);
            const double* adj = side == 0 ? UAb : UBb;
            double mx = 0.0, df = 0.0;
            for (int i = 0; i < NV; ++i) {
                mx = std::fmax(mx, std::fabs(phi.d[i]));
                df = std::fmax(df, std::fabs(phi.d[i] - adj[i]));
            }
            const double rel = df / std::fmax(mx, 1e-300);
            if (rel > worst) worst = rel;
            if (rel > 1e-11) {
                std::printf("mismatch it=%d side=%d rel=%.3e\n", it, side, rel);
                for (int i = 0; i < NV; ++i) std::printf("  fwd %.16e adj %.16e\n", phi.d[i], adj[i]);
                return 1;
            }
        }
        // branch census: upwind side x star region, pStar clamp, shock factors
        {
            const double gm = ph.gamma, Ma = ph.mach, MS = gm * Ma * Ma, G2 = 0.5 * (gm + 1.0) / gm;
            double un[2], pr[2], c[2], r[2] = {UA[0], UB[0]};
            const double* Us[2] = {UA, UB};
            for (int k = 0; k < 2; ++k) {
                double ms = 0.0, unr = 0.0;
                for (int d = 0; d < D; ++d) {
                    ms += Us[k][d + 1] * Us[k][d + 1];
                    unr += Us[k][d + 1] * n[d];
                }
                un[k] = unr / r[k];
                pr[k] = (Us[k][D + 1] - ms / r[k] * (MS * 0.5)) * (gm - 1.0);
                c[k] = std::sqrt(pr[k] / r[k]) / Ma;
            }
            double pS = 0.5 * (pr[0] + pr[1]) - (un[1] - un[0]) * 0.5 * (c[0] + c[1]) * 0.5 * (r[0] + r[1]) * 0.5 * MS;
            if (pS < 0.0) { ++clamps; pS = 0.0; }
            const double qA = pS > pr[0] ? std::sqrt(1.0 + (pS / pr[0] - 1.0) * G2) : 1.0;
            const double qB = pS > pr[1] ? std::sqrt(1.0 + (pS / pr[1] - 1.0) * G2) : 1.0;
            if (pS > pr[0] || pS > pr[1]) ++shocks;
            const double sA = un[0] - c[0] * qA, sB = un[1] + c[1] * qB;
            const double CA = r[0] * (sA - un[0]), CB = r[1] * (sB - un[1]);
            const double S = (CB * un[1] - CA * un[0] + (pr[0] - pr[1]) / MS) / (CB - CA);
            const int left = S > 0.0;
            const int star = left ? (sA <= 0.0) : (sB >= 0.0);
            ++branches[left][star];
        }
    }
    std::printf("worst relative difference %.3e\n", worst);
    std::printf("branches: right/supersonic %d right/star %d left/supersonic %d left/star %d clamp %d shock %d\n",
                branches[0][0], branches[0][1], branches[1][0], branches[1][1], clamps, shocks);
    const bool covered = branches[0][0] && branches[0][1] && branches[1][0] && branches[1][1] && clamps && shocks;
    return (worst <= 1e-11 && covered) ? 0 : 1;
}
