// rb_solve.cuh -- in-group accelerators and the group loop, run by one team (cluster) per problem.
//
// Restates on the device: livolant! (src/tools/livolant.jl:110-154), anderson!
// (src/tools/anderson.jl:38-140), gmres! (src/tools/gmres.jl:35-133), bicgstab!
// (src/tools/bicgstab.jl:30-101), sn_one_speed (sn_one_speed.jl:81-195) and the group loop of
// compute_flux(::SN) (sn_flux.jl:146-224). Every scalar decision (convergence tests,
// Hessenberg, Givens, Anderson normal equations) is taken from team reductions whose bits are
// identical in every thread, so all threads of the cluster branch together; each CTA keeps its
// own copy of the small scalar arrays, updated by its leader thread.
#pragma once
#include <math_constants.h>

#include "rb_kernels.cuh"
#include "rb_local1d.cuh"
#include "rb_sweep_oct.cuh"

namespace rb {

struct SolveStat {
    int iter;
    double resid;
    int conv;
    double rho;
};

__device__ __forceinline__ double rho_estimate(double r0, double r, int it) {  // krylov_state.jl:139-144
    if (it > 1 && r0 > 0.0 && r > 0.0) return pow(r / r0, 1.0 / (it - 1));
    return CUDART_NAN;
}

// LO: the team runs only 1D problems on the local pass (the kernel that carries no other pass)
template <class Team, bool LO = false>
struct Solver {
    Team &t;
    const DevProblem &P;
    GroupShared &gs;
    int ig;
    const double *phiE_in;
    double *phiE_out;
    long long npass;
    void *local = nullptr;  // shared-memory region of the local 1D pass (and of the 3D octant sweep)
    long long local_bytes = 0;
    int local_ok = 0;       // this problem takes the local 1D pass
    int local_w = 0;        // and keeps the slice of w in shared memory in the Gram-Schmidt loop

    __device__ double *vec(int k) const { return P.vecs + (long long)k * P.vstride; }

    // load_and_pass! (sn_one_speed.jl:138-143): out <- T(zin)
    // The mixed form runs every pass with FP32 angular arithmetic except two per group
    // (final = 1), which are FP64: the Krylov right-hand side c = T(0) and the reconstruction
    // pass, which produces the returned flux moments and the energy-face flux carried into the
    // next group (the outer defect-correction update).
    // One copy of the pass per kernel (it is called from every accelerator): its own register
    // allocation, and a compile time that does not grow with the number of call sites.
    __device__ __noinline__ void pass(const double *zin, double *out, int homog, int mv, int final = 0) {
        const int mixed = (P.precision == 1 && !final) ? 1 : 0;
        npass++;
        if constexpr (std::is_same<Team, ClusterTeam>::value) {
            if (LO || local_ok) {
                pass1d_local(t, P, gs, local, zin, out, homog, mv, ig, phiE_in, phiE_out, mixed);
                return;
            }
        }
        if constexpr (std::is_same<Team, GridTeam>::value) {  // the grid team runs 2D/3D problems only
            pass_md(t, P, gs, local, local_bytes, zin, out, homog, mv, ig, phiE_in, phiE_out, mixed);
        } else if constexpr (!LO) {
            if (P.ndims == 1) pass1d(t, P, gs, zin, out, homog, mv, ig, phiE_in, phiE_out, mixed);
            else pass_md(t, P, gs, local, local_bytes, zin, out, homog, mv, ig, phiE_in, phiE_out, mixed);
        }
    }
    __device__ void fixedpoint(double *out, const double *zin) { pass(zin, out, 0, 0); }
    // matvec! (sn_one_speed.jl:147): out <- zin − A·zin
    __device__ void matvec(double *out, const double *zin) { pass(zin, out, 1, 1); }
    __device__ double norm(const double *a) { return sqrt(vdot(t, a, a, P.nstate)); }

    // ---------------------------------------------------------------- livolant (and "none")
    __device__ __noinline__ SolveStat livolant(double *z, int maxit, double tol, int period) {
        const long long N = P.nstate;
        double *g = vec(1), *z1 = vec(3), *z0 = vec(4);
        int nhist = 0, iter = 0, conv = 0;
        double resid = 1.0, resid0 = CUDART_NAN;
        for (int it = 1; it <= maxit; it++) {
            fixedpoint(g, z); iter++;
            // ‖g − z‖ and ‖g‖ in one reduction
            double v[2] = {0.0, 0.0};
            for (long long i = t.rank(); i < N; i += t.size()) {
                const double f = g[i] + (-1.0) * z[i];
                v[0] += f * f; v[1] += g[i] * g[i];
            }
            t.template sumk<2>(v);
            resid = sqrt(v[0]) / fmax(sqrt(v[1]), 1e-16);
            if (isnan(resid0)) resid0 = resid;
            if (resid < tol) { vcopy(t, z, g, N); conv = 1; break; }
            if (period > 0 && it % period == 0 && nhist >= 2) {
                double w[2] = {0.0, 0.0};
                for (long long i = t.rank(); i < N; i += t.size()) {
                    const double e0 = z1[i] - z0[i], e1 = g[i] - z1[i], de = e1 - e0;
                    w[0] += e0 * de; w[1] += de * de;
                }
                t.template sumk<2>(w);
                double mu = 1.0;
                if (w[1] != 0.0) { mu = -w[0] / w[1]; if (mu <= 0) mu = 1.0; }
                for (long long i = t.rank(); i < N; i += t.size()) {
                    z[i] = g[i] * mu + (1.0 - mu) * z1[i];
                    z0[i] = z1[i];
                    z1[i] = g[i];
                }
            } else {
                for (long long i = t.rank(); i < N; i += t.size()) {
                    z[i] = g[i];
                    z0[i] = z1[i];
                    z1[i] = g[i];
                }
            }
            t.sync();
            nhist++;
        }
        SolveStat s = {iter, resid, conv, rho_estimate(resid0, resid, iter)};
        return s;
    }

    // ---------------------------------------------------------------- anderson (β = 1)
    __device__ __noinline__ SolveStat anderson(double *z, int depth, int maxit, double tol) {
        const long long N = P.nstate;
        const int m = depth > 1 ? depth : 1;
        double *g = vec(1), *f = vec(2), *fo = vec(3), *go = vec(4);
        // history ring: logical i -> slot (head + i) % m; ΔF slot s = vec(5+s), ΔG = vec(5+m+s)
        int nh = 0, head = 0, iter = 0, conv = 0;
        double resid = 1.0, resid0 = CUDART_NAN;
        for (int it = 1; it <= maxit; it++) {
            fixedpoint(g, z); iter++;
            double v[3] = {0.0, 0.0, 0.0};
            for (long long i = t.rank(); i < N; i += t.size()) {
                const double fi = g[i] + (-1.0) * z[i];
                f[i] = fi;
                v[0] += fi * fi; v[1] += z[i] * z[i]; v[2] += g[i] * g[i];
            }
            t.template sumk<3>(v);
            resid = sqrt(v[0]) / fmax(fmax(sqrt(v[1]), sqrt(v[2])), 1e-16);
            if (isnan(resid0)) resid0 = resid;
            if (resid < tol) { conv = 1; break; }
            if (it == 1) {
                vaxpy(t, 1.0, f, z, N);
            } else {
                if (nh == m) { head = (head + 1) % m; nh--; }  // popfirst!
                const int slot = (head + nh) % m;
                double *dF = vec(5 + slot), *dG = vec(5 + m + slot);
                for (long long i = t.rank(); i < N; i += t.size()) {
                    dF[i] = f[i] + (-1.0) * fo[i];
                    dG[i] = g[i] + (-1.0) * go[i];
                }
                t.sync();
                nh++;
                const int mk = nh;
                for (int i = 0; i < mk; i++) {
                    const double *dFi = vec(5 + (head + i) % m);
                    double bi = vdot(t, dFi, f, N);
                    if (t.leader()) gs.b[i] = bi;
                    for (int j = 0; j < mk; j++) {
                        double aij = vdot(t, dFi, vec(5 + (head + j) % m), N);
                        if (t.leader()) gs.A[i + mk * j] = aij;
                    }
                }
                __syncthreads();
                if (t.leader()) {
                    double *A = gs.A, *x = gs.b;
                    double tr = 0.0;
                    for (int i = 0; i < mk; i++) tr += A[i + mk * i];
                    const double lam = 1e-12 * (tr / mk + 1e-300);
                    for (int i = 0; i < mk; i++) A[i + mk * i] += lam;
                    const int n = mk;  // anderson_solve (anderson.jl:112-140)
                    for (int k = 0; k < n; k++) {
                        int p = k; double mx = fabs(A[k + n * k]);
                        for (int i = k + 1; i < n; i++) if (fabs(A[i + n * k]) > mx) { mx = fabs(A[i + n * k]); p = i; }
                        if (p != k) {
                            for (int j = k; j < n; j++) { double tt = A[k + n * j]; A[k + n * j] = A[p + n * j]; A[p + n * j] = tt; }
                            double tt = x[k]; x[k] = x[p]; x[p] = tt;
                        }
                        const double piv = A[k + n * k];
                        if (piv == 0.0) continue;
                        for (int i = k + 1; i < n; i++) {
                            const double fac = A[i + n * k] / piv;
                            for (int j = k; j < n; j++) A[i + n * j] -= fac * A[k + n * j];
                            x[i] -= fac * x[k];
                        }
                    }
                    for (int k = n - 1; k >= 0; k--) {
                        double s = x[k];
                        for (int j = k + 1; j < n; j++) s -= A[k + n * j] * x[j];
                        x[k] = A[k + n * k] != 0.0 ? s / A[k + n * k] : 0.0;
                    }
                }
                __syncthreads();
                // z ← z + f − Σ γ_i ΔG_i  (β = 1: the ΔF term carries a zero factor)
                for (long long i = t.rank(); i < N; i += t.size()) {
                    double zi = z[i] + 1.0 * f[i];
                    for (int k = 0; k < mk; k++) zi += -gs.b[k] * vec(5 + m + (head + k) % m)[i];
                    z[i] = zi;
                }
                t.sync();
            }
            for (long long i = t.rank(); i < N; i += t.size()) { fo[i] = f[i]; go[i] = g[i]; }
            t.sync();
        }
        SolveStat s = {iter, resid, conv, rho_estimate(resid0, resid, iter)};
        return s;
    }

    // Modified Gram-Schmidt of w against V_0..V_j for a problem on the local 1D pass: each CTA
    // keeps its slice of w, and of the basis vector in use, in shared memory, so a step reads
    // only the next basis vector from memory. Same steps and fused dot products as the
    // team-wide loop in gmres; writes H[0..j, j] and V_{j+1}, returns false when not local.
    __device__ __noinline__ bool mgs_local(const double *w, int jb, int m, double &hjp1) {
        if constexpr (std::is_same<Team, ClusterTeam>::value) {
            if (!local_w) return false;
            Local1D L(P, t.crank, t.ncta, local);
            double *ws = L.ws, *vs = reinterpret_cast<double *>(L.psi);
            double *H = gs.H;
            {
                const double *V0 = vec(4);
                double acc[1] = {0.0};
                double xw[RB_SVU], xv[RB_SVU];
                RB_SLICE_LOOP(L, { xw[u_] = w[g]; xv[u_] = V0[g]; }, {
                    ws[j] = xw[u_];
                    vs[j] = xv[u_];
                    acc[0] += xw[u_] * xv[u_];
                })
                t.template sumk<1>(acc);
                double h = acc[0];
                for (int i = 0; i <= jb; i++) {
                    if (t.leader()) H[i + (m + 1) * jb] = h;
                    double a1[1] = {0.0};
                    if (i < jb) {
                        const double *Vn = vec(4 + i + 1);
                        double xn[RB_SVU];
                        RB_SLICE_LOOP(L, { xn[u_] = Vn[g]; }, {
                            const double wq = ws[j] + (-h) * vs[j];
                            ws[j] = wq;
                            vs[j] = xn[u_];
                            a1[0] += wq * xn[u_];
                        })
                    } else {
                        RB_SLICE_LOOP(L, {}, {
                            const double wq = ws[j] + (-h) * vs[j];
                            ws[j] = wq;
                            a1[0] += wq * wq;
                        })
                    }
                    t.template sumk<1>(a1);
                    h = a1[0];
                }
                hjp1 = sqrt(h);
                if (hjp1 > 0.0) {
                    const double inv = 1.0 / hjp1;
                    double *Vn = vec(4 + jb + 1);
                    RB_SLICE_LOOP(L, {}, { Vn[g] = ws[j] * inv; })
                }
            }
            return true;
        }
        return false;
    }

    // ---------------------------------------------------------------- gmres(m)
    __device__ __noinline__ SolveStat gmres(double *z, const double *rhs, int restart, int maxit, double tol) {
        const long long N = P.nstate, N2 = P.vstride / 2;  // elements, pairs
        const int m = restart > 1 ? restart : 1;
        SolveStat st = {0, 0.0, 1, CUDART_NAN};
        const double bnorm = sqrt(vdot2(t, rhs, rhs, N2));
        if (bnorm == 0.0) { vzero(t, z, N); return st; }
        double *r = vec(2), *w = vec(3);
        double *H = gs.H;
#define HH(i, j) H[(i) + (m + 1) * (j)]
        int iter = 0, conv = 0;
        double resid = 1.0, resid0 = CUDART_NAN;
        while (iter < maxit && !conv) {
            matvec(r, z); iter++;
            double v1[1] = {0.0};
            {  // r = c − M z
                double2 xc[RB_VU2], xr[RB_VU2];
                const double2 *c2 = RB_CD2(rhs);
                double2 *r2 = RB_D2(r);
                RB_VPAIRS(t, N2, { xc[u_] = c2[q]; xr[u_] = r2[q]; }, {
                    double2 ri;
                    ri.x = xc[u_].x - xr[u_].x;
                    ri.y = xc[u_].y - xr[u_].y;
                    r2[q] = ri;
                    v1[0] += ri.x * ri.x;
                    v1[0] += ri.y * ri.y;
                })
            }
            t.template sumk<1>(v1);
            const double beta = sqrt(v1[0]);
            resid = beta / bnorm;
            if (isnan(resid0)) resid0 = resid;
            if (resid < tol) { conv = 1; break; }
            {
                const double inv = 1.0 / beta;
                double2 *V02 = RB_D2(vec(4));
                const double2 *r2 = RB_CD2(r);
                double2 xr[RB_VU2];
                RB_VPAIRS(t, N2, { xr[u_] = r2[q]; }, { V02[q] = make_double2(xr[u_].x * inv, xr[u_].y * inv); })
            }
            if (t.leader()) {
                for (int i = 0; i <= m; i++) gs.g[i] = 0.0;
                gs.g[0] = beta;
            }
            t.sync();
            int k = 0;
            for (int j = 0; j < m; j++) {
                if (iter >= maxit) break;
                matvec(w, vec(4 + j)); iter++;
                double hjp1;
                if (!mgs_local(w, j, m, hjp1)) {
                // modified Gram-Schmidt, one sweep per basis vector: w ← w − h_i V_i fused with
                // the dot product of the updated w against V_{i+1} (or against itself at the end)
                double h = vdot2(t, w, vec(4), N2);
                double2 *w2 = RB_D2(w);
                for (int i = 0; i <= j; i++) {
                    if (t.leader()) HH(i, j) = h;
                    const double2 *Vi2 = RB_CD2(vec(4 + i));
                    const double2 *Vn2 = (i < j) ? RB_CD2(vec(4 + i + 1)) : nullptr;
                    double acc[1] = {0.0};
                    double2 xw[RB_VU2], xv[RB_VU2], xn[RB_VU2];
                    if (Vn2) {
                        RB_VPAIRS(t, N2, { xw[u_] = w2[q]; xv[u_] = Vi2[q]; xn[u_] = Vn2[q]; }, {
                            double2 wq;
                            wq.x = xw[u_].x + (-h) * xv[u_].x;
                            wq.y = xw[u_].y + (-h) * xv[u_].y;
                            w2[q] = wq;
                            acc[0] += wq.x * xn[u_].x;
                            acc[0] += wq.y * xn[u_].y;
                        })
                    } else {
                        RB_VPAIRS(t, N2, { xw[u_] = w2[q]; xv[u_] = Vi2[q]; }, {
                            double2 wq;
                            wq.x = xw[u_].x + (-h) * xv[u_].x;
                            wq.y = xw[u_].y + (-h) * xv[u_].y;
                            w2[q] = wq;
                            acc[0] += wq.x * wq.x;
                            acc[0] += wq.y * wq.y;
                        })
                    }
                    t.template sumk<1>(acc);
                    h = acc[0];
                }
                hjp1 = sqrt(h);
                if (hjp1 > 0.0) {
                    const double inv = 1.0 / hjp1;
                    double2 *Vn2 = RB_D2(vec(4 + j + 1));
                    double2 xw[RB_VU2];
                    RB_VPAIRS(t, N2, { xw[u_] = w2[q]; }, { Vn2[q] = make_double2(xw[u_].x * inv, xw[u_].y * inv); })
                }
                }
                if (t.leader()) {
                    HH(j + 1, j) = hjp1;
                    for (int i = 0; i < j; i++) {
                        const double temp = gs.cs[i] * HH(i, j) + gs.sn[i] * HH(i + 1, j);
                        HH(i + 1, j) = -gs.sn[i] * HH(i, j) + gs.cs[i] * HH(i + 1, j);
                        HH(i, j) = temp;
                    }
                    const double denom = hypot(HH(j, j), HH(j + 1, j));
                    if (denom == 0.0) { gs.cs[j] = 1.0; gs.sn[j] = 0.0; }
                    else { gs.cs[j] = HH(j, j) / denom; gs.sn[j] = HH(j + 1, j) / denom; }
                    HH(j, j) = gs.cs[j] * HH(j, j) + gs.sn[j] * HH(j + 1, j);
                    HH(j + 1, j) = 0.0;
                    gs.g[j + 1] = -gs.sn[j] * gs.g[j];
                    gs.g[j] = gs.cs[j] * gs.g[j];
                }
                t.sync();
                k = j + 1;
                resid = fabs(gs.g[j + 1]) / bnorm;
                if (resid < tol) { conv = 1; break; }
                if (hjp1 == 0.0) break;
            }
            if (t.leader()) {
                for (int i = k - 1; i >= 0; i--) {
                    double s = gs.g[i];
                    for (int l = i + 1; l < k; l++) s -= HH(i, l) * gs.y[l];
                    gs.y[i] = HH(i, i) != 0.0 ? s / HH(i, i) : 0.0;
                }
            }
            __syncthreads();
            // z += Σ y_i V_i, in basis order per element
            {
                double2 xz[RB_VU2];
                double2 *z2 = RB_D2(z);
                RB_VPAIRS(t, N2, { xz[u_] = z2[q]; }, {
                    double2 zq = xz[u_];
                    for (int i = 0; i < k; i++) {
                        const double2 v = RB_CD2(vec(4 + i))[q];
                        zq.x += gs.y[i] * v.x;
                        zq.y += gs.y[i] * v.y;
                    }
                    z2[q] = zq;
                })
            }
            t.sync();
            if (conv) break;
        }
#undef HH
        st.iter = iter; st.resid = resid; st.conv = conv; st.rho = rho_estimate(resid0, resid, iter);
        return st;
    }

    // ---------------------------------------------------------------- bicgstab
    // Vector loops over 16-byte element pairs of CTA-contiguous slices (the pad element of an odd
    // state stays zero in every vector): 8 pairs in flight per thread over two vectors, 4 over
    // three or four.
    __device__ __noinline__ SolveStat bicgstab(double *z, const double *rhs, int maxit, double tol) {
        const long long N = P.nstate, N2 = P.vstride / 2;
        SolveStat st = {0, 0.0, 1, CUDART_NAN};
        const double bnorm = sqrt(vdot2(t, rhs, rhs, N2));
        if (bnorm == 0.0) { vzero(t, z, N); return st; }
        double *r = vec(2), *rh = vec(3), *p = vec(4), *v = vec(5), *s = vec(6), *tt = vec(7);
        double2 *r2 = RB_D2(r), *rh2 = RB_D2(rh), *p2 = RB_D2(p), *v2 = RB_D2(v), *s2 = RB_D2(s), *z2 = RB_D2(z);
        const double2 *c2 = RB_CD2(rhs), *t2 = RB_CD2(tt);
        const double2 zero2 = make_double2(0.0, 0.0);
        matvec(r, z);
        double a1[1] = {0.0};
        {
            double2 xc[RB_VU2], xr[RB_VU2];
            RB_VPAIRS(t, N2, { xc[u_] = c2[q]; xr[u_] = r2[q]; }, {
                const double2 ri = make_double2(xc[u_].x - xr[u_].x, xc[u_].y - xr[u_].y);
                r2[q] = ri; rh2[q] = ri; p2[q] = zero2; v2[q] = zero2;
                a1[0] += ri.x * ri.x;
                a1[0] += ri.y * ri.y;
            })
        }
        t.template sumk<1>(a1);
        int iter = 1, conv = 0;
        double resid = sqrt(a1[0]) / bnorm, resid0 = resid;
        if (resid < tol) { st.iter = iter; st.resid = resid; st.conv = 1; st.rho = CUDART_NAN; return st; }
        double rho_old = 1.0, alpha = 1.0, omega = 1.0;
        const double tiny = 1e-300;
        // (r̂·r) of the coming iteration: the initial loop's Σ r² (r̂ = r there), then the last
        // loop's second sum (the same terms, in the same order per thread, as a separate dot)
        double rho_next = a1[0];
        while (iter < maxit) {
            const double rho_new = rho_next;
            if (fabs(rho_new) < tiny) break;
            const double beta = (rho_new / rho_old) * (alpha / omega);
            {
                double2 xr[4], xp[4], xv[4];
                RB_VPAIRS_D(t, N2, 4, { xr[u_] = r2[q]; xp[u_] = p2[q]; xv[u_] = v2[q]; }, {
                    p2[q] = make_double2(xr[u_].x + 1.0 * (beta * (xp[u_].x + (-omega) * xv[u_].x)),
                                         xr[u_].y + 1.0 * (beta * (xp[u_].y + (-omega) * xv[u_].y)));
                })
            }
            t.sync();
            matvec(v, p); iter++;
            const double denom = vdot2(t, rh, v, N2);
            if (fabs(denom) < tiny) break;
            alpha = rho_new / denom;
            double a2[1] = {0.0};
            {
                double2 xr[RB_VU2], xv[RB_VU2];
                RB_VPAIRS(t, N2, { xr[u_] = r2[q]; xv[u_] = v2[q]; }, {
                    const double2 si = make_double2(xr[u_].x + (-alpha) * xv[u_].x, xr[u_].y + (-alpha) * xv[u_].y);
                    s2[q] = si;
                    a2[0] += si.x * si.x;
                    a2[0] += si.y * si.y;
                })
            }
            t.template sumk<1>(a2);
            const double sn_ = sqrt(a2[0]);
            if (sn_ / bnorm < tol) {
                vaxpy(t, alpha, p, z, N);
                resid = sn_ / bnorm;
                conv = 1;
                break;
            }
            matvec(tt, s); iter++;
            double a3[2] = {0.0, 0.0};
            {
                double2 xt[RB_VU2], xs[RB_VU2];
                RB_VPAIRS(t, N2, { xt[u_] = t2[q]; xs[u_] = s2[q]; }, {
                    a3[0] += xt[u_].x * xt[u_].x;
                    a3[0] += xt[u_].y * xt[u_].y;
                    a3[1] += xt[u_].x * xs[u_].x;
                    a3[1] += xt[u_].y * xs[u_].y;
                })
            }
            t.template sumk<2>(a3);
            if (a3[0] < tiny) break;
            omega = a3[1] / a3[0];
            double a4[2] = {0.0, 0.0};
            {
                double2 xz[4], xp[4], xs[4], xt[4], xh[4];
                RB_VPAIRS_D(t, N2, 4, { xz[u_] = z2[q]; xp[u_] = p2[q]; xs[u_] = s2[q]; xt[u_] = t2[q]; xh[u_] = rh2[q]; }, {
                    z2[q] = make_double2((xz[u_].x + alpha * xp[u_].x) + omega * xs[u_].x,
                                         (xz[u_].y + alpha * xp[u_].y) + omega * xs[u_].y);
                    const double2 ri = make_double2(xs[u_].x + (-omega) * xt[u_].x, xs[u_].y + (-omega) * xt[u_].y);
                    r2[q] = ri;
                    a4[0] += ri.x * ri.x;
                    a4[0] += ri.y * ri.y;
                    a4[1] += xh[u_].x * ri.x;
                    a4[1] += xh[u_].y * ri.y;
                })
            }
            t.template sumk<2>(a4);
            rho_next = a4[1];
            resid = sqrt(a4[0]) / bnorm;
            if (resid < tol) { conv = 1; break; }
            if (fabs(omega) < tiny) break;
            rho_old = rho_new;
        }
        st.iter = iter; st.resid = resid; st.conv = conv; st.rho = rho_estimate(resid0, resid, iter);
        return st;
    }

    // ---------------------------------------------------------------- sn_one_speed
    __device__ __noinline__ SolveStat one_speed(double *flux_g) {
        const long long N = P.nstate, nphi = P.nphi;
        const long long nE = (long long)P.nd * P.nm4 * P.ncell;
        // zero-source short-circuit (sn_one_speed.jl:115-120)
        int any = 0;
        for (int f = 0; f < 2 * P.ndims; f++) {
            const double *src = P.surf[f];
            if (!src) continue;
            for (long long k = t.rank(); k < (long long)P.np_source * P.fcells[f / 2]; k += t.size())
                if (src[ig + (long long)P.ng * k] != 0.0) any = 1;
        }
        for (long long i = t.rank(); i < nphi; i += t.size()) if (P.qlout[i] != 0.0) any = 1;
        if (P.csd) for (long long i = t.rank(); i < nE; i += t.size()) if (phiE_in[i] != 0.0) any = 1;
        any = t.any(any);
        if (!any) {
            for (long long i = t.rank(); i < nphi; i += t.size()) flux_g[i] = 0.0;
            if (P.csd) for (long long i = t.rank(); i < nE; i += t.size()) phiE_out[i] = 0.0;
            t.sync();
            SolveStat s = {1, 0.0, 1, CUDART_NAN};
            return s;
        }
        double *z = vec(0);
        vzero(t, z, N);  // initial state: 𝚽l of the group = 0, boundary in-moments = 0
        SolveStat st;
        const bool mixed = P.precision == 1;
        if (P.accel == 0 || P.accel == 1) {
            st = livolant(z, P.maxit, mixed ? fmax(P.tol, RB_MIXED_TOL) : P.tol, P.accel == 0 ? 0 : 3);
        } else if (P.accel == 2) {
            st = anderson(z, P.depth, P.maxit, mixed ? fmax(P.tol, RB_MIXED_TOL) : P.tol);
        } else {
            double *rhs = vec(1);
            pass(z, rhs, 0, 0, 1);  // c = T(0), FP64 in both forms
            // The mixed form solves with the FP32 operator to RB_MIXED_TOL1, then takes one outer
            // defect-correction step: the residual r = c − (I − A)·z with the FP64 operator, the
            // correction δ from the FP32-operator solve of (I − A)·δ = r to the tolerance that
            // brings the whole residual to `tol`, z ← z + δ.
            const double tol1 = mixed ? fmax(P.tol, RB_MIXED_TOL1) : P.tol;
            if (P.accel == 3) st = gmres(z, rhs, P.restart, P.maxit, tol1);
            else st = bicgstab(z, rhs, P.maxit, tol1);
            if (mixed) {
                double *dz = vec(P.nvec - 2), *res = vec(P.nvec - 1);
                pass(z, res, 1, 1, 1);  // res = z − A·z, FP64
                double v[2] = {0.0, 0.0};
                for (long long i = t.rank(); i < N; i += t.size()) {
                    const double ri = rhs[i] - res[i];
                    res[i] = ri;
                    v[0] += ri * ri;
                    v[1] += rhs[i] * rhs[i];
                }
                t.template sumk<2>(v);
                const double rel = v[1] > 0.0 ? sqrt(v[0] / v[1]) : 0.0;
                if (rel >= P.tol) {
                    vzero(t, dz, N);
                    const double tol2 = fmax(P.tol / rel, RB_MIXED_TOL);
                    SolveStat s2;
                    if (P.accel == 3) s2 = gmres(dz, res, P.restart, P.maxit, tol2);
                    else s2 = bicgstab(dz, res, P.maxit, tol2);
                    vaxpy(t, 1.0, dz, z, N);
                    st.iter += s2.iter + 1;
                    st.resid = s2.resid * rel;
                    st.conv = s2.conv;
                } else {
                    st.iter += 1;
                    st.resid = rel;
                    st.conv = 1;
                }
            }
        }
        // reconstruction pass (sn_one_speed.jl:184-187)
        double *out = vec(1);
        pass(z, out, 0, 0, 1);
        vcopy(t, flux_g, out, nphi);
        return st;
    }
};

// ------------------------------------------------------------------------------------------
// the group loop of compute_flux(::SN) for one problem (sn_flux.jl:146-224)
// ------------------------------------------------------------------------------------------
template <class Team, bool LO = false>
__device__ void solve_problem(Team &t, const DevProblem &P, GroupShared &gs, void *local = nullptr,
                              long long local_bytes = 0) {
    const int local_ok = (local && local1d_ok(P, (int)t.ncta, local_bytes)) ? 1 : 0;
    const int local_w = (local && local1d_w(P, (int)t.ncta, local_bytes)) ? 1 : 0;
    const int ng = P.ng, nmat = P.nmat, np = P.np, nd = P.nd, nm = P.nm5;
    const long long nphi = P.nphi, ncell = P.ncell;
    const long long nE = (long long)nd * P.nm4 * ncell;
    const int st_ = P.solver_type;
    double *phiE_in = P.phiE_a, *phiE_out = P.phiE_b;
    // the pad element of each Krylov vector (odd nstate) starts and stays zero
    if (P.vstride > P.nstate)
        for (int k = t.rank(); k < P.nvec; k += t.size()) P.vecs[(long long)k * P.vstride + P.nstate] = 0.0;
    if (P.csd) { vzero(t, phiE_in, nE); vzero(t, phiE_out, nE); }
    // the octant sweep's progress flags count up from zero within this solve
    if (P.ndims == 3)
        for (int k = t.rank(); k < RB_OCT_MAXCTA; k += t.size()) P.oct_flags[k] = 0ull;
    if (threadIdx.x == 0) gs.oct_epoch = 0;
    t.sync();
    long long npass = 0;
    for (int ig = 0; ig < ng; ig++) {
        // per-group constants, one copy per CTA
        for (int m = threadIdx.x; m < nmat; m += blockDim.x) {
            gs.sigt[m] = P.sigma_t[ig + (long long)ng * m];
            if (P.csd) {
                const double dE = P.e_width[ig];
                gs.sm[m] = P.s_minus[ig + (long long)ng * m] / dE;
                gs.sp[m] = P.s_plus[ig + (long long)ng * m] / dE;
            } else {
                gs.sm[m] = gs.sp[m] = 0.0;
            }
            gs.tg[m] = (st_ == 2 || st_ == 4) ? P.t_mom[ig + (long long)ng * m] : 0.0;
        }
        __syncthreads();
        if (P.csd) {  // CSD block of the cell matrix: Σ_w (S_w/ΔE)·K_w + (S⁺/ΔE)·B
            const int nn = nm * nm;
            for (long long o = t.rank(); o < (long long)nmat * nn; o += t.size()) {
                const int m = (int)(o / nn), e = (int)(o % nn);
                const double dE = P.e_width[ig];
                double v = gs.sp[m] * P.Bcsd[e];
                for (int w = 0; w < P.oE; w++)
                    v += (P.s_mom[ig + (long long)ng * (m + (long long)nmat * w)] / dE) * P.Kcsd[(long long)w * nn + e];
                P.scsd[o] = v;
            }
        }
        // ys[m][p] = Σs_in[m, pl[p]]: the in-group scattering source of moment p (zero for the
        // solvers without it, sn_inner_pass.jl:21); T[m] scales the Fokker-Planck product
        const bool scat = (st_ != 4 && st_ != 5 && st_ != 6);
        for (long long o = t.rank(); o < (long long)nmat * np; o += t.size()) {
            const int p = (int)(o % np);
            const int m = (int)(o / np);
            P.kmat[o] = scat ? P.sigma_s[m + (long long)nmat * (ig + (long long)ng * (ig + (long long)ng * P.pl[p]))] : 0.0;
        }
        // Qlout = Σ_{gi≠ig} Σs[mat,gi,ig,l]·𝚽[gi] + volume source (scattering_source.jl:59-68;
        // groups above ig are still zero in the single outer iteration, sn_flux.jl:150,157)
        for (long long o = t.rank(); o < nphi; o += t.size()) {
            const int p = (int)(o % np);
            const long long c = o / ((long long)np * nm);
            const int m = P.mat[c];
            double q = 0.0;
            if (st_ != 4 && st_ != 5) {
                const double *ss = P.sigma_s + m + (long long)nmat * (long long)ng * (ig + (long long)ng * P.pl[p]);
                for (int gi = 0; gi < ig; gi++) q += ss[(long long)nmat * gi] * P.flux[(long long)gi * nphi + o];
            }
            // the volume source: particle source + fixed source (transport.jl:89-90)
            if (P.pvol || P.vol) {
                double vs = P.pvol ? P.pvol[(long long)ig * nphi + o] : 0.0;
                if (P.vol) vs = vs + P.vol[(long long)ig * nphi + o];
                q += vs;
            }
            P.qlout[o] = q;
        }
        if (P.csd && ig != 0) {  // 𝚽E12 .* ΔE[ig] / ΔE[ig-1]
            const double r1 = P.e_width[ig], r0 = P.e_width[ig - 1];
            for (long long i = t.rank(); i < nE; i += t.size()) phiE_in[i] = phiE_in[i] * r1 / r0;
        }
        t.sync();
        if constexpr (std::is_same<Team, ClusterTeam>::value) {
            if (LO || local_ok) {
                Local1D L(P, t.crank, t.ncta, local);
                local1d_group_setup(P, L);
                local1d_factor_fixed(P, gs, L);
            }
        }
        // Mn·Qlout into ψ, then kept as Qnout for the passes of this group
        m2d_tiles(t, P, gs, P.qlout, nullptr, 0);
        t.sync();
        vcopy(t, P.qnout, P.psi, (long long)nd * nm * ncell);
        Solver<Team, LO> S{t, P, gs, ig, phiE_in, phiE_out, 0};
        S.local = local;
        S.local_bytes = local ? local_bytes : 0;
        S.local_ok = local_ok;
        S.local_w = local_w;
        SolveStat s = S.one_speed(P.flux + (long long)ig * nphi);
        npass += S.npass;
        if (t.rank() == 0) {
            P.rho[ig] = s.rho; P.resid[ig] = s.resid; P.iters[ig] = s.iter; P.conv[ig] = s.conv;
            if (!s.conv) atomicOr(P.status, RB_DEV_NOT_CONVERGED);
        }
        double *tmp = phiE_in; phiE_in = phiE_out; phiE_out = tmp;
        t.sync();
    }
    // 𝚽cutoff[p,is,c] = Σ_n Dn[p,n]·𝚽E12[n,is,c] for is < Nm4 (sn_flux.jl:215-218)
    if (P.csd) {
        for (long long o = t.rank(); o < nphi; o += t.size()) {
            const int p = (int)(o % np);
            const int is = (int)((o / np) % nm);
            const long long c = o / ((long long)np * nm);
            double s = 0.0;
            if (is < P.nm4)
                for (int n = 0; n < nd; n++)
                    s += P.dn[p + (long long)np * n] * phiE_in[n + (long long)nd * (is + (long long)P.nm4 * c)];
            P.cutoff[o] = s;
        }
    }
    if (t.rank() == 0) *P.passes = npass;
    t.sync();
}

// ------------------------------------------------------------------------------------------
// the persistent kernels (each defined in its own translation unit, rb_kernel_*.cu)
// ------------------------------------------------------------------------------------------
// Dynamic shared memory: GroupShared, then `local_bytes` for the local 1D pass (and the 3D
// octant sweep). Clusters pull problems from the work queue `queue`.
__global__ void __launch_bounds__(RB_THREADS, 1) solve_batch_kernel(DevProblem *const *probs, int nprob, int *queue,
                                                                 int local_bytes);
// The same loop for batches whose every problem takes the local 1D pass: the kernel carries no
// other pass, so its registers go to that path alone.
__global__ void __launch_bounds__(RB_THREADS, 1) solve_local1d_kernel(DevProblem *const *probs, int nprob, int *queue,
                                                                   int local_bytes);
// One large (2D/3D) problem on the whole GPU: a cooperative launch, one team of every CTA.
__global__ void __launch_bounds__(RB_THREADS, 1) solve_grid_kernel(DevProblem *prob, double *gpart, int local_bytes);

}  // namespace rb
