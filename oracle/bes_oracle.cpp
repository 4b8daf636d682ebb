/*
 * bes_oracle.cpp -- TEST INFRASTRUCTURE.  CPU oracle of the coupled
 * Keller-Miksis ensemble integrator (see bes_oracle.h for the reference
 * files and line ranges each part restates).  Never linked into the product.
 *
 * Arithmetic order.  The reference leaves fused multiply-add contraction to
 * nvcc, which the oracle cannot observe, so the oracle fixes one explicit
 * order (every fma below is written out; compile with -ffp-contract=off):
 *   - sums over units (dot products, the transposed product, the residual
 *     maximum) use the reference's halving tree (Steppers.cuh:709-805) over
 *     the units padded with zeros to P = max(32, next power of two >= N);
 *     for N >= 32 this is exactly the reference's order, for N < 32 it is the
 *     correct sum (the reference's reduction is wrong there: it returns
 *     2*s[0] because nP2Warps = 0);
 *   - the direct products (coupling value, A*x0, A*p; Steppers.cuh:576-584,
 *     :647-666, :683-688, which accumulate columns 0..N-1 in one chain)
 *     use four interleaved fma chains over the columns j = 0, 1, 2, 3 mod 4,
 *     combined as (s0 + s1) + (s2 + s3) (a shorter dependency chain on the
 *     GPU); A*p adds that sum to p_i;
 *   - the operator element is W_ij = (rD_i * C_ij) * X1sq_j (Steppers.cuh:685).
 *   - shared-matrix association (systems with N > 32 whose coupling matrix is
 *     shared by the launch and staged once in shared memory): the products
 *     apply C to a scaled vector instead of forming W,
 *       A x0:  rD_i * sum_j C_ij (X1sq_j x0_j)        (fma chains as above)
 *       A p:   p_i + rD_i * sum_j C_ij (X1sq_j p_j)
 *       A^T p~: p~_i + X1sq_i * tree_j C_ji (rD_j p~_j).
 * The product kernel follows the same order, so oracle and kernel agree
 * bit for bit.
 */
#include "bes_oracle.h"
#include "oracle_math.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

/* solves of the single-reduction recurrence redone with the reference's (diagnostics) */
std::atomic<long long> g_rec1_fallbacks{0};
std::atomic<long long> g_rec1_fallback_capped{0};
using std::fma;
const int UD = BES_ORACLE_UD;
const int NUP = BES_ORACLE_NUP;
const int NCOLL = BES_ORACLE_NCOLL;
const int NUA = BES_ORACLE_NUA;
const int NIUA = BES_ORACLE_NIUA;
const double PI = 3.14159265358979323846;

/* ---------------------------------------------------------------------------
 * Keller-Miksis right-hand side, BubbleEnsemble_SystemDefinition.cuh:8-49.
 * F0 = X1, F1 = N/D (uncoupled acceleration), CPT = -2 X0 X1^2, CPF = 1/D. */
inline void km_ode(double X0, double X1, double T, const double* u,
                   double* F0, double* F1, double* CPT, double* CPF) {
    double rx1 = 1.0 / X0;
    double p = oracle_math::pow_recip(X0, u[10]);   /* (1/X0)^u10 */
    double s1, c1;
    oracle_math::sincospi(2.0 * T, &s1, &c1);
    double s2, c2;
    if (u[11] == 0.0 && u[12] == 0.0) {
        s2 = 0.0; c2 = 1.0;              /* sin(0), cos(0) of the second harmonic */
    } else {
        double arg = fma(2.0 * u[11] * PI, T, u[12]);
        oracle_math::sincos(arg, &s2, &c2);
    }
    double g = fma(u[9], X1, 1.0);                       /* 1 + u9 X1 */
    double N = fma(u[1], X1, u[0]) * p;                  /* (u0 + u1 X1) p */
    N = fma(-u[2], g, N);                                /* - u2 (1 + u9 X1) */
    N = fma(-u[3], rx1, N);                              /* - u3 / X0 */
    N = fma(-(u[4] * X1), rx1, N);                       /* - u4 X1 / X0 */
    double h = fma(-0.5 * u[9], X1, 1.5);                /* 1.5 (1 - u9 X1 / 3) */
    N = fma(-(h * X1), X1, N);                           /* - 1.5 (1 - u9 X1/3) X1^2 */
    double sd = fma(u[6], s2, u[5] * s1);
    N = fma(-sd, g, N);                                  /* - (u5 s1 + u6 s2)(1 + u9 X1) */
    double cd = fma(u[8], c2, u[7] * c1);
    N = fma(-X0, cd, N);                                 /* - X0 (u7 c1 + u8 c2) */
    double D = fma(u[4], u[9], fma(-(u[9] * X0), X1, X0)); /* X0 - u9 X0 X1 + u4 u9 */
    double rD = 1.0 / D;
    *F0 = X1;
    *F1 = N * rD;
    *CPT = (-2.0 * X0 * X1) * X1;
    *CPF = rD;
}

/* four interleaved fma chains over the columns, combined as (s0 + s1) + (s2 + s3) */
template <class A, class B>
inline double row_sum4(int n, A a, B b) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j = 0; j < n; j++) s[j & 3] = fma(a(j), b(j), s[j & 3]);
    return (s[0] + s[1]) + (s[2] + s[3]);
}

inline int next_pow2_32(int n) {
    int p = 32;
    while (p < n) p *= 2;
    return p;
}

/* halving-tree sum of v[0..n) padded with zeros to P (Steppers.cuh:745-774) */
inline double tree_sum(const double* v, int n, double* tmp) {
    int P = next_pow2_32(n);
    for (int i = 0; i < P; i++) tmp[i] = i < n ? v[i] : 0.0;
    for (int L = P / 2; L >= 1; L /= 2)
        for (int i = 0; i < L; i++) tmp[i] = tmp[i] + tmp[i + L];
    return tmp[0];
}

inline double tree_max(const double* v, int n, double* tmp) {
    int P = next_pow2_32(n);
    for (int i = 0; i < P; i++) tmp[i] = i < n ? v[i] : 0.0;
    for (int L = P / 2; L >= 1; L /= 2)
        for (int i = 0; i < L; i++) tmp[i] = std::fmax(tmp[i], tmp[i + L]);
    return tmp[0];
}

struct Work {
    int N;
    std::vector<double> cpt, rd, x1sq, xu, b, r, rt, p, pt, q, qt, x, W, tmp, tmp2, us, vs, z, zt, wv, wtv, r0, tmp3;
    explicit Work(int n) : N(n) {
        int P = next_pow2_32(n);
        cpt.resize(n); rd.resize(n); x1sq.resize(n); xu.resize(n); b.resize(n);
        r.resize(n); rt.resize(n); p.resize(n); pt.resize(n); q.resize(n); qt.resize(n);
        x.resize(n); W.resize((size_t)n * n); tmp.resize(P); tmp2.resize(n); us.resize(n); vs.resize(n);
        z.resize(n); zt.resize(n); wv.resize(n); wtv.resize(n); r0.resize(n); tmp3.resize(n);
    }
};

/* ---------------------------------------------------------------------------
 * Coupled right-hand side for all units of one system:
 * OdeFunction_WithBiConjugateGradient, Steppers.cuh:432-562.
 * y0/y1: states of the N units; up: per-unit parameter pointers (stride `ups`).
 * Writes f0/f1; returns completed BiCG iterations; sets *capped when the
 * iteration limit was used up without meeting an exit test. */
int coupled_rhs(Work& w, double T, const double* y0, const double* y1,
                const double* up, long ups, const double* C, int max_iter,
                double* f0, double* f1, bool* capped, bool shared_assoc = false,
                const double* ra = nullptr, const double* cb = nullptr, bool symmetric = false, int variant = 0,
                int bw = 0) {
    const int N = w.N;
    /* banded association (banded storage, bw > 0, and no shared-matrix
     * association): only the wrapping band j = i + d - bw (mod N),
     * d = 0 .. nd - 1, nd = min(2 bw + 1, N), of C is read (with nd = N every
     * column exactly once), with four chains over d (d mod 4); W is kept by
     * diagonal, Wb[d][i] = W[i][j(i, d)], and the transposed product of unit i
     * sums Wb[d][k] vt[k] over k = i + bw - d (mod N) */
    const bool band = bw > 0 && !shared_assoc;
    const int nd = std::min(2 * bw + 1, N);
    auto jband = [&](int i, int d) { return (((i + d - bw) % N) + N) % N; };
    auto band_sum4 = [&](auto term) {
        double c[4] = {0.0, 0.0, 0.0, 0.0};
        for (int d = 0; d < nd; d++) term(d, c[d & 3]);
        return (c[0] + c[1]) + (c[2] + c[3]);
    };
    double upl[NUP];
    for (int i = 0; i < N; i++) {
        for (int k = 0; k < NUP; k++) upl[k] = up[(long)k * ups + i];
        km_ode(y0[i], y1[i], T, upl, &f0[i], &w.xu[i], &w.cpt[i], &w.rd[i]);
        w.x1sq[i] = y0[i] * y0[i];
    }
    if (shared_assoc) {
        /* C = diag(a) G diag(b): u = b X1sq before G, v = rD a after G (a = b = 1 without factors) */
        for (int i = 0; i < N; i++) {
            w.us[i] = (cb ? cb[i] : 1.0) * w.x1sq[i];
            w.vs[i] = w.rd[i] * (ra ? ra[i] : 1.0);
            w.tmp2[i] = (cb ? cb[i] : 1.0) * w.cpt[i];
        }
    }
    /* b = rD (C CPT) + x_u ; r = b - A x_u  (Steppers.cuh:495-505, :576-584, :647-666) */
    for (int i = 0; i < N; i++) {
        double bi, ax;
        if (band) {
            bi = band_sum4([&](int d, double& acc) { const int j = jband(i, d); acc = fma(C[i + (long)j * N], w.cpt[j], acc); });
            bi = fma(w.rd[i], bi, w.xu[i]);
            ax = band_sum4([&](int d, double& acc) {
                const int j = jband(i, d);
                acc = fma(C[i + (long)j * N] * w.x1sq[j], w.xu[j], acc);
            });
            ax = fma(w.rd[i], ax, w.xu[i]);
            w.b[i] = bi;
            w.r[i] = bi - ax;
            w.rt[i] = w.r[i];
            w.x[i] = w.xu[i];
            for (int d = 0; d < nd; d++) {
                const int j = jband(i, d);
                w.W[i + (long)d * N] = (w.rd[i] * C[i + (long)j * N]) * w.x1sq[j];   /* Wb[d][i] */
            }
            continue;
        }
        if (shared_assoc) {
            bi = row_sum4(N, [&](int j) { return C[i + (long)j * N]; }, [&](int j) { return w.tmp2[j]; });
            bi = fma(w.vs[i], bi, w.xu[i]);
            ax = row_sum4(N, [&](int j) { return C[i + (long)j * N]; }, [&](int j) { return w.us[j] * w.xu[j]; });
            ax = fma(w.vs[i], ax, w.xu[i]);
        } else {
            bi = row_sum4(N, [&](int j) { return C[i + (long)j * N]; }, [&](int j) { return w.cpt[j]; });
            bi = fma(w.rd[i], bi, w.xu[i]);
            ax = row_sum4(N, [&](int j) { return C[i + (long)j * N] * w.x1sq[j]; }, [&](int j) { return w.xu[j]; });
            ax = fma(w.rd[i], ax, w.xu[i]);
        }
        w.b[i] = bi;
        w.r[i] = bi - ax;
        w.rt[i] = w.r[i];
        w.x[i] = w.xu[i];
        for (int j = 0; j < N; j++) w.W[i + (long)j * N] = (w.rd[i] * C[i + (long)j * N]) * w.x1sq[j];
    }
    /* q = A v (row sums) and qt = A^T vt (tree sums or, for a symmetric shared
     * matrix, row sums), Steppers.cuh:669-706 */
    auto apply = [&](const double* v, const double* vt, double* q, double* qt) {
        if (band) {
            for (int i = 0; i < N; i++) {
                q[i] = v[i] + band_sum4([&](int d, double& acc) { acc = fma(w.W[i + (long)d * N], v[jband(i, d)], acc); });
                qt[i] = vt[i] + band_sum4([&](int d, double& acc) {
                    const int k = (((i + bw - d) % N) + N) % N;
                    acc = fma(w.W[k + (long)d * N], vt[k], acc);
                });
            }
            return;
        }
        if (shared_assoc) {
            for (int j = 0; j < N; j++) { w.z[j] = w.us[j] * v[j]; w.zt[j] = w.vs[j] * vt[j]; }
        }
        for (int i = 0; i < N; i++) {
            if (shared_assoc) {
                double s = row_sum4(N, [&](int j) { return C[i + (long)j * N]; }, [&](int j) { return w.z[j]; });
                q[i] = fma(w.vs[i], s, v[i]);
                if (symmetric) {
                    /* C = C^T: the transposed product as a row sum (the kernel reads each entry once for both) */
                    double st = row_sum4(N, [&](int j) { return C[i + (long)j * N]; }, [&](int j) { return w.zt[j]; });
                    qt[i] = fma(w.us[i], st, vt[i]);
                } else {
                    for (int j = 0; j < N; j++) w.tmp2[j] = C[j + (long)i * N] * w.zt[j];
                    qt[i] = fma(w.us[i], tree_sum(w.tmp2.data(), N, w.tmp.data()), vt[i]);
                }
            } else {
                q[i] = v[i] + row_sum4(N, [&](int j) { return w.W[i + (long)j * N]; }, [&](int j) { return v[j]; });
                for (int j = 0; j < N; j++) w.tmp2[j] = w.W[j + (long)i * N] * vt[j];
                qt[i] = vt[i] + tree_sum(w.tmp2.data(), N, w.tmp.data());
            }
        }
    };
    int done = 0;
    bool exited = false;
    /* the reference's recurrence, Steppers.cuh:508-561 */
    auto reference_recurrence = [&]() {
        for (int i = 0; i < N; i++) w.tmp2[i] = w.r[i] * w.rt[i];
        double rho1 = tree_sum(w.tmp2.data(), N, w.tmp.data());
        double rho2 = 0.0;
        for (int iter = 1; iter <= max_iter; iter++) {
            if (iter == 1) {
                for (int i = 0; i < N; i++) { w.p[i] = w.r[i]; w.pt[i] = w.rt[i]; }
                if (std::fabs(rho1) < 1e-6) { exited = true; break; }
            } else {
                double beta = rho1 / rho2;
                for (int i = 0; i < N; i++) {
                    w.p[i] = fma(beta, w.p[i], w.r[i]);
                    w.pt[i] = fma(beta, w.pt[i], w.rt[i]);
                }
            }
            apply(w.p.data(), w.pt.data(), w.q.data(), w.qt.data());
            for (int i = 0; i < N; i++) w.tmp2[i] = w.pt[i] * w.q[i];
            double alpha = rho1 / tree_sum(w.tmp2.data(), N, w.tmp.data());
            for (int i = 0; i < N; i++) {
                w.x[i] = fma(alpha, w.p[i], w.x[i]);
                w.r[i] = fma(-alpha, w.q[i], w.r[i]);
                w.rt[i] = fma(-alpha, w.qt[i], w.rt[i]);
            }
            for (int i = 0; i < N; i++) w.tmp2[i] = std::fabs(w.r[i]);
            double rmax = tree_max(w.tmp2.data(), N, w.tmp.data());
            rho2 = rho1;
            done++;
            if (rmax < 1e-6) { exited = true; break; }
            for (int i = 0; i < N; i++) w.tmp2[i] = w.r[i] * w.rt[i];
            rho1 = tree_sum(w.tmp2.data(), N, w.tmp.data());
        }
    };
    if (variant == 0) {
        reference_recurrence();
    } else {
        /* Single-reduction recurrence (the same iterates in exact arithmetic):
         * the products of the residuals w = A r, w~ = A^T r~ come first, then
         * one reduction gives rho = r.r~ and mu = r~.w together, and
         *   beta = rho / rho_prev,  sigma = mu - beta^2 sigma_prev,
         *   p = r + beta p, p~ = r~ + beta p~, q = w + beta q, q~ = w~ + beta q~,
         *   alpha = rho / sigma,
         * so that q = A p, q~ = A^T p~ and sigma = p~.A p (the two cross terms
         * of p~.A p equal -rho/alpha_prev each by the biorthogonality of the
         * residuals, and rho/alpha_prev = beta sigma_prev).  The exits are the
         * reference's: |rho| < 1e-6 before the first update, max |r| < 1e-6
         * after each update, at most max_iter updates.
         * Its q is a recurrence, not a product, so r can drift from the true
         * residual (and sigma can collapse): the solution is accepted only when
         * every x is finite and the true residual b - A x passes the reference's
         * exit test (max < 1e-6), or when the first rho test ended the solve;
         * otherwise the solve is redone from the start with the reference's
         * recurrence. */
        for (int i = 0; i < N; i++) w.r0[i] = w.r[i];
        double sigma = 0.0, rho_prev = 0.0;
        for (int iter = 1; iter <= max_iter; iter++) {
            apply(w.r.data(), w.rt.data(), w.wv.data(), w.wtv.data());
            for (int i = 0; i < N; i++) w.tmp2[i] = w.r[i] * w.rt[i];
            const double rho = tree_sum(w.tmp2.data(), N, w.tmp.data());
            for (int i = 0; i < N; i++) w.tmp2[i] = w.rt[i] * w.wv[i];
            const double mu = tree_sum(w.tmp2.data(), N, w.tmp.data());
            if (iter == 1) {
                if (std::fabs(rho) < 1e-6) { exited = true; break; }
                for (int i = 0; i < N; i++) {
                    w.p[i] = w.r[i]; w.pt[i] = w.rt[i]; w.q[i] = w.wv[i]; w.qt[i] = w.wtv[i];
                }
                sigma = mu;
            } else {
                const double beta = rho / rho_prev;
                sigma = fma(-(beta * beta), sigma, mu);
                for (int i = 0; i < N; i++) {
                    w.p[i] = fma(beta, w.p[i], w.r[i]);
                    w.pt[i] = fma(beta, w.pt[i], w.rt[i]);
                    w.q[i] = fma(beta, w.q[i], w.wv[i]);
                    w.qt[i] = fma(beta, w.qt[i], w.wtv[i]);
                }
            }
            const double alpha = rho / sigma;
            rho_prev = rho;
            for (int i = 0; i < N; i++) {
                w.x[i] = fma(alpha, w.p[i], w.x[i]);
                w.r[i] = fma(-alpha, w.q[i], w.r[i]);
                w.rt[i] = fma(-alpha, w.qt[i], w.rt[i]);
            }
            for (int i = 0; i < N; i++) w.tmp2[i] = std::fabs(w.r[i]);
            const double rmax = tree_max(w.tmp2.data(), N, w.tmp.data());
            done++;
            if (rmax < 1e-6) { exited = true; break; }
        }
        /* an exit at the first rho test leaves x = x_u, as the reference's recurrence does */
        bool accept = exited;
        for (int i = 0; i < N && accept; i++) accept = std::isfinite(w.x[i]);
        if (accept && done > 0) {
            /* true residual b - A x (the second product's result is not used) */
            for (int i = 0; i < N; i++) w.tmp3[i] = 0.0;
            apply(w.x.data(), w.tmp3.data(), w.wv.data(), w.wtv.data());
            for (int i = 0; i < N; i++) w.tmp2[i] = std::fabs(w.b[i] - w.wv[i]);
            accept = tree_max(w.tmp2.data(), N, w.tmp.data()) < 1e-6;
        }
        if (!accept) {
            g_rec1_fallbacks++;
            if (!exited) g_rec1_fallback_capped++;
            exited = false;
            for (int i = 0; i < N; i++) { w.r[i] = w.r0[i]; w.rt[i] = w.r0[i]; w.x[i] = w.xu[i]; }
            reference_recurrence();
        }
    }
    *capped = !exited;
    for (int i = 0; i < N; i++) f1[i] = w.x[i];
    return done;
}

/* ---------------------------------------------------------------------------
 * One system, one or more periods. */
struct SystemRun {
    const bes_oracle_problem* P;
    int s, N;
    long off, tot;
    Work w;
    std::vector<double> y0, y1, yn0, yn1, e0, e1, k[6][2], s0, s1, ev_a, ev_n, uacc;
    std::vector<int> iuacc;
    SystemRun(const bes_oracle_problem* p, int sid)
        : P(p), s(sid), N(p->units[sid]), off(p->unit_offset[sid]), tot(p->total_units), w(p->units[sid]) {
        y0.resize(N); y1.resize(N); yn0.resize(N); yn1.resize(N); e0.resize(N); e1.resize(N);
        for (auto& kk : k) { kk[0].resize(N); kk[1].resize(N); }
        s0.resize(N); s1.resize(N); ev_a.resize(N); ev_n.resize(N);
        uacc.resize((size_t)N * NUA); iuacc.resize((size_t)N * NIUA);
        for (int i = 0; i < N; i++) {
            y0[i] = p->state[off + i];
            y1[i] = p->state[tot + off + i];
            for (int kk = 0; kk < NUA; kk++) uacc[(size_t)i * NUA + kk] = p->uacc[(long)kk * tot + off + i];
            for (int kk = 0; kk < NIUA; kk++) iuacc[(size_t)i * NIUA + kk] = p->iuacc[(long)kk * tot + off + i];
        }
    }
    void write_back() {
        for (int i = 0; i < N; i++) {
            P->state[off + i] = y0[i];
            P->state[tot + off + i] = y1[i];
            for (int kk = 0; kk < NUA; kk++) P->uacc[(long)kk * tot + off + i] = uacc[(size_t)i * NUA + kk];
            for (int kk = 0; kk < NIUA; kk++) P->iuacc[(long)kk * tot + off + i] = iuacc[(size_t)i * NIUA + kk];
        }
    }
    const double* up() const { return P->upar + off; }
    const double* C() const { return P->coupling + P->coupling_offset[s]; }
    bool symmetric_C = false;   /* the system's matrix equals its transpose exactly */
    void find_symmetry() {
        const double* c = C();
        bool sym = true;
        for (int i = 0; i < N && sym; i++)
            for (int j = i + 1; j < N && sym; j++) sym = c[i + (long)j * N] == c[j + (long)i * N];
        symmetric_C = sym;
    }

    int rhs(double T, const double* a0, const double* a1, double* f0, double* f1, int64_t& nbicg, bool& capped_any) {
        bool capped = false;
        int it = coupled_rhs(w, T, a0, a1, up(), tot, C(), P->bicg_max_iter, f0, f1, &capped,
                             P->shared_assoc != 0 && (N > 32 || symmetric_C),
                             P->coupling_row_scale ? P->coupling_row_scale + off : nullptr,
                             P->coupling_col_scale ? P->coupling_col_scale + off : nullptr, symmetric_C,
                             P->bicg_variant, P->band_width);
        nbicg += it;
        if (capped) capped_any = true;
        return it;
    }

    /* RKCK45 stepper, Steppers.cuh:94-425: fills yn, err; returns finiteness */
    bool step_rkck45(double T, double dt, int64_t& nbicg, int64_t& nrhs, bool& capped) {
        auto& K = k;
        rhs(T, y0.data(), y1.data(), K[0][0].data(), K[0][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) st[i] = fma(K[0][c][i] * (1.0 / 5.0), dt, y[i]);
        }
        rhs(fma(1.0 / 5.0, dt, T), s0.data(), s1.data(), K[1][0].data(), K[1][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) {
                double S = K[0][c][i] * (3.0 / 40.0);
                S = fma(K[1][c][i], 9.0 / 40.0, S);
                st[i] = fma(S, dt, y[i]);
            }
        }
        rhs(fma(3.0 / 10.0, dt, T), s0.data(), s1.data(), K[2][0].data(), K[2][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) {
                double S = K[0][c][i] * (3.0 / 10.0);
                S = fma(K[1][c][i], -9.0 / 10.0, S);
                S = fma(K[2][c][i], 6.0 / 5.0, S);
                st[i] = fma(S, dt, y[i]);
            }
        }
        rhs(fma(3.0 / 5.0, dt, T), s0.data(), s1.data(), K[3][0].data(), K[3][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) {
                double S = K[0][c][i] * (-11.0 / 54.0);
                S = fma(K[1][c][i], 5.0 / 2.0, S);
                S = fma(K[2][c][i], -70.0 / 27.0, S);
                S = fma(K[3][c][i], 35.0 / 27.0, S);
                st[i] = fma(S, dt, y[i]);
            }
        }
        rhs(T + dt, s0.data(), s1.data(), K[4][0].data(), K[4][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) {
                double S = K[0][c][i] * (1631.0 / 55296.0);
                S = fma(K[1][c][i], 175.0 / 512.0, S);
                S = fma(K[2][c][i], 575.0 / 13824.0, S);
                S = fma(K[3][c][i], 44275.0 / 110592.0, S);
                S = fma(K[4][c][i], 253.0 / 4096.0, S);
                st[i] = fma(S, dt, y[i]);
            }
        }
        rhs(fma(7.0 / 8.0, dt, T), s0.data(), s1.data(), K[5][0].data(), K[5][1].data(), nbicg, capped);
        nrhs += 6;
        bool finite = true;
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* yn = c == 0 ? yn0.data() : yn1.data();
            double* er = c == 0 ? e0.data() : e1.data();
            for (int i = 0; i < N; i++) {
                double S = K[0][c][i] * (37.0 / 378.0);
                S = fma(K[2][c][i], 250.0 / 621.0, S);
                S = fma(K[3][c][i], 125.0 / 594.0, S);
                S = fma(K[5][c][i], 512.0 / 1771.0, S);
                yn[i] = fma(S, dt, y[i]);
                double E = K[0][c][i] * (37.0 / 378.0 - 2825.0 / 27648.0);
                E = fma(K[2][c][i], 250.0 / 621.0 - 18575.0 / 48384.0, E);
                E = fma(K[3][c][i], 125.0 / 594.0 - 13525.0 / 55296.0, E);
                E = fma(K[4][c][i], 0.0 - 277.0 / 14336.0, E);
                E = fma(K[5][c][i], 512.0 / 1771.0 - 1.0 / 4.0, E);
                er[i] = fma(dt, std::fabs(E), 1e-18);
                if (!std::isfinite(yn[i]) || !std::isfinite(er[i])) finite = false;
            }
        }
        return finite;
    }

    /* classical RK4 (no reference stepper exists; the reference ships only its
     * fixed-step controller, ErrorControllers.cuh:424-450) */
    bool step_rk4(double T, double dt, int64_t& nbicg, int64_t& nrhs, bool& capped) {
        auto& K = k;
        rhs(T, y0.data(), y1.data(), K[0][0].data(), K[0][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) st[i] = fma(K[0][c][i] * 0.5, dt, y[i]);
        }
        rhs(fma(0.5, dt, T), s0.data(), s1.data(), K[1][0].data(), K[1][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) st[i] = fma(K[1][c][i] * 0.5, dt, y[i]);
        }
        rhs(fma(0.5, dt, T), s0.data(), s1.data(), K[2][0].data(), K[2][1].data(), nbicg, capped);
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* st = c == 0 ? s0.data() : s1.data();
            for (int i = 0; i < N; i++) st[i] = fma(K[2][c][i], dt, y[i]);
        }
        rhs(T + dt, s0.data(), s1.data(), K[3][0].data(), K[3][1].data(), nbicg, capped);
        nrhs += 4;
        bool finite = true;
        for (int c = 0; c < 2; c++) {
            const double* y = c == 0 ? y0.data() : y1.data();
            double* yn = c == 0 ? yn0.data() : yn1.data();
            for (int i = 0; i < N; i++) {
                double S = K[0][c][i] * (1.0 / 6.0);
                S = fma(K[1][c][i], 1.0 / 3.0, S);
                S = fma(K[2][c][i], 1.0 / 3.0, S);
                S = fma(K[3][c][i], 1.0 / 6.0, S);
                yn[i] = fma(S, dt, y[i]);
                if (!std::isfinite(yn[i])) finite = false;
            }
        }
        return finite;
    }

    /* collapse bookkeeping callbacks, BubbleEnsemble_SystemDefinition.cuh:79-105 */
    void after_event(int i) {
        int& c = iuacc[(size_t)i * NIUA];
        c++;
        if (c < NCOLL) {
            uacc[(size_t)i * NUA + c] = y0[i];
            uacc[(size_t)i * NUA + c + NCOLL] = y0[i];
        }
    }
    void after_step(int i) {
        int c = iuacc[(size_t)i * NIUA];
        if (c < NCOLL && y0[i] < uacc[(size_t)i * NUA + c + NCOLL]) uacc[(size_t)i * NUA + c + NCOLL] = y0[i];
    }

    void store_dense(int& idx, int update_do, int update, int& skipped, double& do_time, double T, double TD1) {
        const bes_oracle_problem* p = P;
        if (update_do == 1 && idx < p->ndo) {
            for (int i = 0; i < N; i++) {
                p->dense_state[(long)idx * UD * tot + off + i] = y0[i];
                p->dense_state[(long)idx * UD * tot + tot + off + i] = y1[i];
            }
            p->dense_time[(long)idx * p->n_systems + s] = T;
        }
        if (update_do == 1) {
            idx++;
            skipped = 0;
            do_time = std::fmin(T + p->do_min_dt, TD1);
        }
        if (update_do == 0 && update == 1) skipped++;
    }

    /* One Solve() of the reference: Solver.cuh:82-130 (set-up), :262-325
     * (initialisation, first event values, first dense store), :329-572
     * (step loop), :599-648 (write-back). */
    void period() {
        const bes_oracle_problem* p = P;
        const double TD0 = p->time_domain[s];
        const double TD1 = p->time_domain[p->n_systems + s];
        double T = p->actual_time[s];
        double dt = p->dt0, newdt = p->dt0;
        int ndo = p->ndo;
        int do_idx = ndo > 0 ? p->dense_index[s] : 0;
        int update_do = 1, skipped = 0;
        double do_time = 0.0;
        int terminate = 0, udt = 0;
        double rtol[UD], atol[UD];
        for (int c = 0; c < UD; c++) {
            rtol[c] = p->rtol[(long)c * p->n_systems + s];
            atol[c] = p->atol[(long)c * p->n_systems + s];
        }
        /* Initialization callback: unit 0 sets T = TD[0] (SystemDefinition:108-116) */
        T = TD0;
        for (int i = 0; i < N; i++) ev_a[i] = y1[i];   /* EventFunction: EF = X1 */
        if (ndo > 0) store_dense(do_idx, update_do, 1, skipped, do_time, T, TD1);
        const double tol = p->event_tol;
        const int dir = p->event_dir;
        int64_t attempted = 0;
        while (!terminate) {
            int update = 1, end = 0;
            dt = newdt;
            if (dt > (TD1 - T)) { dt = TD1 - T; end = 1; }
            if (attempted >= p->max_steps_per_period) {
                p->status[s] |= BES_ORACLE_ST_STEP_BUDGET;
                break;
            }
            attempted++;
            if (p->min_dt && dt < p->min_dt[s]) p->min_dt[s] = dt;
            bool capped = false;
            bool finite = p->algorithm == 1 ? step_rkck45(T, dt, p->n_bicg_iter[s], p->n_rhs[s], capped)
                                             : step_rk4(T, dt, p->n_bicg_iter[s], p->n_rhs[s], capped);
            if (capped) p->status[s] |= BES_ORACLE_ST_BICG_CAP;
            if (p->algorithm == 1) {
                /* ErrorController_RKCK45, ErrorControllers.cuh:454-542 */
                double relerr = 1e30;
                int upd = 1;
                for (int i = 0; i < N; i++) {
                    double rr = 1e30;
                    int ru = 1;
                    for (int c = 0; c < UD; c++) {
                        double yn = c == 0 ? yn0[i] : yn1[i];
                        double yo = c == 0 ? y0[i] : y1[i];
                        double er = c == 0 ? e0[i] : e1[i];
                        double et = std::fmax(rtol[c] * std::fmax(std::fabs(yn), std::fabs(yo)), atol[c]);
                        ru = ru & (er < et);
                        rr = std::fmin(rr, et / er);
                    }
                    upd &= ru;
                    relerr = std::fmin(relerr, rr);
                }
                update = upd;
                double mult = update == 1 ? 0.8 * oracle_math::pow(relerr, 1.0 / 5.0)
                                          : 0.8 * oracle_math::pow(relerr, 1.0 / 4.0);
                if (!std::isfinite(mult)) finite = false;
                if (!finite) {
                    mult = p->shrink;
                    update = 0;
                    if (dt < p->dtmin * 1.01) {
                        p->status[s] |= BES_ORACLE_ST_NONFINITE;
                        terminate = 1;
                    }
                } else if (dt < p->dtmin * 1.01) {
                    p->status[s] |= BES_ORACLE_ST_MIN_STEP;
                    update = 1;
                }
                mult = std::fmin(mult, p->grow);
                mult = std::fmax(mult, p->shrink);
                newdt = dt * mult;
                newdt = std::fmin(newdt, p->dtmax);
                newdt = std::fmax(newdt, p->dtmin);
            } else {
                /* ErrorController_RK4, ErrorControllers.cuh:424-450 */
                if (!finite) {
                    p->status[s] |= BES_ORACLE_ST_NONFINITE;
                    terminate = 1;
                    update = 0;
                }
                newdt = p->dt0;
            }
            if (!terminate) {
                for (int i = 0; i < N; i++) ev_n[i] = yn1[i];
                if (update == 1) {
                    /* EventTimeStepControl, EventHandling.cuh:216-268 */
                    double evdt = dt;
                    int corrected = 0;
                    for (int i = 0; i < N; i++) {
                        double a = ev_a[i], n = ev_n[i];
                        if ((a > tol && n < -tol && dir <= 0) || (a < -tol && n > tol && dir >= 0)) {
                            double cand = (-a) / (n - a) * dt;
                            if (cand < evdt) evdt = cand;
                            corrected = 1;
                        }
                    }
                    if (corrected) {
                        if (evdt < p->dtmin) {
                            p->status[s] |= BES_ORACLE_ST_EVENT_MISSED;
                        } else {
                            newdt = evdt;
                            update = 0;
                        }
                    }
                }
            }
            if (update == 1) {
                T += dt;
                for (int i = 0; i < N; i++) { y0[i] = yn0[i]; y1[i] = yn1[i]; }
                p->n_accepted[s]++;
                for (int i = 0; i < N; i++) after_step(i);
                for (int i = 0; i < N; i++) {
                    double a = ev_a[i], n = ev_n[i];
                    if ((a > tol && std::fabs(n) < tol && dir <= 0) || (a < -tol && std::fabs(n) < tol && dir >= 0))
                        after_event(i);
                }
                for (int i = 0; i < N; i++) ev_a[i] = y1[i];
            } else {
                p->n_rejected[s]++;
            }
            if (ndo > 0) {
                /* DenseOutputStorageCondition, DenseOutput.cuh:372-395 */
                if (update == 1) {
                    update_do = (do_idx < ndo && do_time < T && skipped >= (p->do_save_frequency - 1)) ? 1 : 0;
                    if (do_idx < ndo && (end == 1 || udt == 1)) update_do = 1;
                } else {
                    update_do = 0;
                }
                store_dense(do_idx, update_do, update, skipped, do_time, T, TD1);
            }
            if (update == 1 && (end == 1 || udt == 1)) terminate = 1;
        }
        p->actual_time[s] = T;
        if (ndo > 0) p->dense_index[s] = do_idx;
    }
};

}  // namespace

extern "C" {

int bes_oracle_solve(const bes_oracle_problem* p, int n_periods, int reset_at,
                     const double* uacc_reset, const int32_t* iuacc_reset, int n_threads) {
    if (!p || p->n_systems < 0) return 1;
    int nsys = std::min(p->n_systems, p->active_systems);
#ifdef _OPENMP
    if (n_threads <= 0) n_threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
#endif
    for (int s = 0; s < nsys; s++) {
        SystemRun run(p, s);
        run.find_symmetry();
        for (int per = 0; per < n_periods; per++) {
            if (per == reset_at) {
                for (int i = 0; i < run.N; i++) {
                    for (int kk = 0; kk < NUA; kk++) run.uacc[(size_t)i * NUA + kk] = uacc_reset[kk];
                    for (int kk = 0; kk < NIUA; kk++) run.iuacc[(size_t)i * NIUA + kk] = iuacc_reset[kk];
                }
            }
            run.period();
        }
        run.write_back();
    }
    return 0;
}

double bes_oracle_pow(double x, double y) { return oracle_math::pow(x, y); }
double bes_oracle_pow_recip(double x, double y) { return oracle_math::pow_recip(x, y); }
double bes_oracle_exp(double x) { return oracle_math::exp(x); }
double bes_oracle_log(double x) { return oracle_math::log(x); }
void bes_oracle_sincospi(double x, double* s, double* c) { oracle_math::sincospi(x, s, c); }
void bes_oracle_sincos(double x, double* s, double* c) { oracle_math::sincos(x, s, c); }

int bes_oracle_rhs(int n, double t, const double* state, const double* upar,
                   const double* coupling, int bicg_max_iter, double* f) {
    Work w(n);
    bool capped = false;
    return coupled_rhs(w, t, state, state + n, upar, n, coupling, bicg_max_iter, f, f + n, &capped);
}

long long bes_oracle_rec1_fallbacks(int reset) {
    const long long v = g_rec1_fallbacks.load();
    if (reset) g_rec1_fallbacks = 0;
    return v;
}

long long bes_oracle_rec1_fallbacks_capped(int reset) {
    const long long v = g_rec1_fallback_capped.load();
    if (reset) g_rec1_fallback_capped = 0;
    return v;
}

int bes_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
