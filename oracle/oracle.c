/*
 * oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C (FP64, OpenMP) restatement of the reference's augmented-Lagrangian inner-loop kernels
 * (Yahiahu/Lagbound, src/lagbound/_core/alm_vcs.py and vcsops.py).  It is the checker for the CUDA path and the
 * timed CPU baseline; only tests/, __graft_entry__.smoke() and bench.py's CPU legs may load it.  The product
 * library (lagbound_b200/) never links or calls it.
 *
 * Every function follows one reference function; the citation is given at each.  Per-row arithmetic keeps the
 * reference's operation order (sequential k-loop dot products, no FMA contraction: build with -ffp-contract=off),
 * so per-row results are bit-identical to the reference's Numba kernels; reductions over rows are summed in row
 * order (the reference's parallel reductions may round differently in the last bits).
 *
 * Conventions: V/X/out are row-major n x k FP64; index arrays are int64 like the reference, VCS columns int32
 * (vcsops.py VCSLevel.set_ws).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;
typedef int32_t i32;

/* alm_vcs.py:528-535 spmm: out = A X */
void orc_spmm(i64 n, i64 k, const i64 *indptr, const i64 *indices, const double *data, const double *X,
              double *out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (i64 i = 0; i < n; i++) {
        double *o = out + i * k;
        for (i64 c = 0; c < k; c++) o[c] = 0.0;
        for (i64 e = indptr[i]; e < indptr[i + 1]; e++) {
            const double w = data[e];
            const double *x = X + indices[e] * k;
            for (i64 c = 0; c < k; c++) o[c] += w * x[c];
        }
    }
}

/* alm_vcs.py:463-474 quadA: sum_ij A_ij v_i.v_j; row partials summed in row order */
double orc_quadA(i64 n, i64 k, const i64 *indptr, const i64 *indices, const double *data, const double *V,
                 double *rowbuf) {
#pragma omp parallel for schedule(dynamic, 64)
    for (i64 i = 0; i < n; i++) {
        double s = 0.0;
        const double *vi = V + i * k;
        for (i64 e = indptr[i]; e < indptr[i + 1]; e++) {
            const double *vj = V + indices[e] * k;
            double dt = 0.0;
            for (i64 c = 0; c < k; c++) dt += vi[c] * vj[c];
            s += data[e] * dt;
        }
        rowbuf[i] = s;
    }
    double tot = 0.0;
    for (i64 i = 0; i < n; i++) tot += rowbuf[i];
    return tot;
}

/* alm_vcs.py:511-526 cluster_sums (one thread): out[lab_i] += d_i v_i in row order (out zeroed here) */
void orc_cluster_sums(i64 n, i64 k, const i64 *lab, const double *d, const double *V, i64 P, double *out) {
    memset(out, 0, sizeof(double) * P * k);
    for (i64 i = 0; i < n; i++) {
        const double di = d[i];
        double *o = out + lab[i] * k;
        for (i64 c = 0; c < k; c++) o[c] += di * V[i * k + c];
    }
}

/* d^T V in row order (alm_vcs.py:1368, 1499: z = d @ V) */
void orc_dTV(i64 n, i64 k, const double *d, const double *V, double *z) {
    for (i64 c = 0; c < k; c++) z[c] = 0.0;
    for (i64 i = 0; i < n; i++)
        for (i64 c = 0; c < k; c++) z[c] += d[i] * V[i * k + c];
}

/* Pair-level Gram matrix H = Y Y^T - diag(dsq) with sequential dot products (alm_vcs.py:1504, 1313-1314). */
void orc_pair_H(i64 P, i64 k, const double *Y, const double *dsq, double *H) {
#pragma omp parallel for schedule(static)
    for (i64 Q = 0; Q < P; Q++)
        for (i64 R = 0; R < P; R++) {
            double h = 0.0;
            for (i64 c = 0; c < k; c++) h += Y[Q * k + c] * Y[R * k + c];
            if (R == Q) h -= dsq[Q];
            H[Q * P + R] = h;
        }
}

/* alm_vcs.py:476-496 level_aug (ne_split off): pp = max(0, sig - rr h), h = sym(H), rr = rho rq_Q rq_R w;
 * returns sum (pp^2 - sig^2)/(2 rr) (row partials summed in row order) and #(h < -1e-9). */
double orc_level_aug(i64 P, const double *H, const double *sig, const double *rq, double w, double rho, double *pp,
                     i64 *nviol) {
    double tot = 0.0;
    i64 cnt = 0;
    for (i64 Q = 0; Q < P; Q++) {
        double s = 0.0;
        i64 c = 0;
        for (i64 R = 0; R < P; R++) {
            const double h = 0.5 * (H[Q * P + R] + H[R * P + Q]);
            const double rr = rho * ((rq[Q] * rq[R]) * w), sg = sig[Q * P + R];
            double p = sg - rr * h;
            if (p < 0.0) p = 0.0;
            pp[Q * P + R] = p;
            s += (p * p - sg * sg) / (2 * rr);
            if (h < -1e-9) c++;
        }
        tot += s;
        cnt += c;
    }
    *nviol = cnt;
    return tot;
}

/* alm_vcs.py:498-509 tri_aug: gt = 1 - tau, pt = max(0, lam - rt gt); returns sum (pt^2 - lam^2)/(2 rt), min gt */
double orc_tri_aug(i64 T, i64 k, const i64 *TI, const double *V, const double *lam, double rt, double *gt, double *pt,
                   double *gmin_out) {
#pragma omp parallel for schedule(static)
    for (i64 t = 0; t < T; t++) {
        const double *va = V + TI[3 * t] * k, *vb = V + TI[3 * t + 1] * k, *vc = V + TI[3 * t + 2] * k;
        double s = 0.0;
        for (i64 q = 0; q < k; q++) s += va[q] * vb[q] + vb[q] * vc[q] - va[q] * vc[q];
        const double g = 1.0 - s;
        gt[t] = g;
        double p = lam[t] - rt * g;
        if (p < 0.0) p = 0.0;
        pt[t] = p;
    }
    double tot = 0.0, gmin = INFINITY;
    for (i64 t = 0; t < T; t++) {
        tot += (pt[t] * pt[t] - lam[t] * lam[t]) / (2 * rt);
        if (gt[t] < gmin) gmin = gt[t];
    }
    *gmin_out = gmin;
    return tot;
}

/* alm_vcs.py:94-104 incidence: row-CSR of triangle corners, code = 3 t + role, in triangle order per row */
void orc_incidence(i64 n, i64 T, const i64 *TI, i64 *ptr, i64 *codes) {
    memset(ptr, 0, sizeof(i64) * (n + 1));
    for (i64 t = 0; t < T; t++)
        for (int r = 0; r < 3; r++) ptr[TI[3 * t + r] + 1]++;
    for (i64 i = 0; i < n; i++) ptr[i + 1] += ptr[i];
    i64 *pos = (i64 *)malloc(sizeof(i64) * (n > 0 ? n : 1));
    memcpy(pos, ptr, sizeof(i64) * n);
    for (i64 t = 0; t < T; t++)
        for (int r = 0; r < 3; r++) {
            const i64 i = TI[3 * t + r];
            codes[pos[i]++] = 3 * t + r;
        }
    free(pos);
}

/* alm_vcs.py:106-120 tri_apply: out += T(w) V, T(w) = sum_t w_t/2 (-E_ab - E_bc + E_ac) (sym.), b = centre */
void orc_tri_apply(i64 n, i64 k, const i64 *TI, const double *w, const i64 *ptr, const i64 *codes, const double *V,
                   double *out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (i64 i = 0; i < n; i++) {
        double *o = out + i * k;
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const i64 code = codes[e], t = code / 3, r = code % 3;
            const double h = 0.5 * w[t];
            if (h == 0.0) continue;
            const double *va = V + TI[3 * t] * k, *vb = V + TI[3 * t + 1] * k, *vc = V + TI[3 * t + 2] * k;
            if (r == 0)
                for (i64 q = 0; q < k; q++) o[q] += h * (vc[q] - vb[q]);
            else if (r == 1)
                for (i64 q = 0; q < k; q++) o[q] -= h * (va[q] + vc[q]);
            else
                for (i64 q = 0; q < k; q++) o[q] += h * (va[q] - vb[q]);
        }
    }
}

/* vcsops.py:246-288 _vcs_aug_rows: per working-set entry pp = max(0, sig - rho r g), value partials, slack flags,
 * next-sweep stZ (stn) when dost; trow/nrow are per-row partials (value, #(g < -1e-9)). */
void orc_vcs_aug(i64 n, i64 k, const double *V, const double *d, const i64 *lab, const double *Y, const i64 *ptr,
                 const i32 *col, const double *sig, const double *rq, double wv, double rho, double *pp,
                 uint8_t *slack, double *stn, int dost, double *trow, i64 *nrow) {
#pragma omp parallel for schedule(dynamic, 64)
    for (i64 i = 0; i < n; i++) {
        const double di = d[i];
        const i64 Ri = lab[i];
        double acc = 0.0;
        i64 cc = 0;
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const i64 R = col[e];
            double s = 0.0;
            for (i64 c = 0; c < k; c++) s += V[i * k + c] * Y[R * k + c];
            double g = di * s;
            if (R == Ri) g = di * (s - di);
            const double sg = sig[e];
            double p = sg;
            if (di > 0.0) {
                const double rr = rho * (wv * rq[R] / (di * di));
                p = sg - rr * g;
                if (p < 0.0) p = 0.0;
                acc += (p * p - sg * sg) / (2 * rr);
            }
            pp[e] = p;
            if (dost) {
                if (rho <= 0.0 || di <= 0.0)
                    stn[e] = p;
                else {
                    const double q = p - rho * (wv * rq[R] / (di * di)) * g;
                    stn[e] = q > 0.0 ? q : 0.0;
                }
            }
            slack[e] = (p == 0.0 && g > 0.0) ? 1 : 0;
            if (g < -1e-9) cc++;
        }
        trow[i] = acc;
        nrow[i] = cc;
    }
}

/* vcsops.py:316-320 vcs_apply (sparse VC operator, matrix-free): out += 1/2 d (S (W X) + (S^T d X)[lab]) - own d^2 X
 * YX = W X (P x k, cluster sums of d_i x_i), ZX = S^T (d X) accumulated in row order (scipy CSR^T semantics). */
void orc_vcs_apply(i64 n, i64 k, i64 P, const double *X, const double *d, const i64 *lab, const i64 *ptr,
                   const i32 *col, const double *sig, const i64 *own, double *out, double *YX, double *ZX) {
    orc_cluster_sums(n, k, lab, d, X, P, YX);
    memset(ZX, 0, sizeof(double) * P * k);
    for (i64 i = 0; i < n; i++)
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const double s = sig[e];
            double *z = ZX + (i64)col[e] * k;
            for (i64 c = 0; c < k; c++) z[c] += s * (d[i] * X[i * k + c]);
        }
#pragma omp parallel for schedule(dynamic, 64)
    for (i64 i = 0; i < n; i++) {
        const double di = d[i];
        const double ow = own[i] >= 0 ? sig[own[i]] : 0.0;
        for (i64 c = 0; c < k; c++) {
            double sy = 0.0;
            for (i64 e = ptr[i]; e < ptr[i + 1]; e++) sy += sig[e] * YX[(i64)col[e] * k + c];
            out[i * k + c] += 0.5 * di * (sy + ZX[lab[i] * k + c]) - (ow * di * di) * X[i * k + c];
        }
    }
}

/* vcsops.py:94-108 vcs_sigt: effective multipliers at (V, Y) for every working-set entry (rho = 0: sig) */
void orc_vcs_sigt(i64 n, i64 k, const double *V, const double *d, const i64 *lab, const double *Y, const i64 *ptr,
                  const i32 *col, const double *sig, const double *rq, double wv, double rho, double *out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (i64 i = 0; i < n; i++) {
        const double di = d[i];
        const i64 Ri = lab[i];
        if (rho <= 0.0 || di <= 0.0) {
            for (i64 e = ptr[i]; e < ptr[i + 1]; e++) out[e] = sig[e];
            continue;
        }
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const i64 R = col[e];
            double s = 0.0;
            for (i64 c = 0; c < k; c++) s += V[i * k + c] * Y[R * k + c];
            const double g = (R == Ri) ? di * (s - di) : di * s;
            const double p = sig[e] - rho * (wv * rq[R] / (di * di)) * g;
            out[e] = p > 0.0 ? p : 0.0;
        }
    }
}

/* vcsops.py:216-235 vcs_zinit_rows: Z_R = sum stZ_e d_i v_i (rows ascending), cnt_R = #(stZ_e > 0) */
void orc_vcs_zinit(i64 n, i64 k, i64 P, const double *V, const double *d, const i64 *ptr, const i32 *col,
                   const double *stZ, double *Z, double *cnt) {
    memset(Z, 0, sizeof(double) * P * k);
    memset(cnt, 0, sizeof(double) * P);
    for (i64 i = 0; i < n; i++) {
        const double f = d[i];
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const i64 R = col[e];
            const double s = stZ[e];
            if (s != 0.0)
                for (i64 c = 0; c < k; c++) Z[R * k + c] += s * (f * V[i * k + c]);
            if (s > 0.0) cnt[R] += 1.0;
        }
    }
}

/* vcsops.py:127-156 vcs_pre: GX += VC half-gradient, KX += VC curvature for the batch rows (useY2 = true) */
void orc_vcs_pre(i64 nr, const i64 *rows, i64 k, const double *V, const double *d, const i64 *lab, const double *Y,
                 const double *Y2, const i64 *ptr, const i32 *col, const double *sig, const double *stZ,
                 const i64 *own, const double *Z, const double *cnt, const double *rq, double wv, double rho,
                 double kap2, double *GX, double *KX) {
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 idx = 0; idx < nr; idx++) {
        const i64 i = rows[idx], Ri = lab[i];
        const double di = d[i];
        double acc[1024];
        double kap = 0.0, pown = 0.0;
        for (i64 c = 0; c < k; c++) acc[c] = 0.0;
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const i64 R = col[e];
            double s = 0.0, p;
            for (i64 c = 0; c < k; c++) s += V[i * k + c] * Y[R * k + c];
            if (rho > 0.0 && di > 0.0) {
                const double g = (R == Ri) ? di * (s - di) : di * s;
                const double rr = wv * rq[R] / (di * di);
                p = sig[e] - rho * rr * g;
                if (p > 0.0) {
                    double y2 = Y2[R];
                    if (R == Ri) y2 = y2 - 2 * di * s + di * di;
                    kap += rho * rr * di * di * y2;
                } else
                    p = 0.0;
            } else
                p = sig[e];
            if (R == Ri) pown = p;
            if (p != 0.0)
                for (i64 c = 0; c < k; c++) acc[c] += p * Y[R * k + c];
        }
        const i64 eo = own[i];
        const double sz = eo >= 0 ? stZ[eo] : 0.0;
        for (i64 c = 0; c < k; c++)
            GX[idx * k + c] += 0.5 * di * (acc[c] - pown * di * V[i * k + c]) + 0.5 * di * (Z[Ri * k + c] - sz * di * V[i * k + c]);
        if (rho > 0.0) kap += kap2 * rho * di * di * wv * rq[Ri] * (cnt[Ri] - (sz > 0.0 ? 1.0 : 0.0));
        KX[idx] += kap;
    }
}

/* vcsops.py:159-164 vcs_yupd + alm_vcs.py:430-438 _acc_rows: aggregate updates in batch-row order */
void orc_acc_rows(i64 nr, const i64 *rows, i64 k, const double *DD, double *z, i64 nl, i64 n, const i64 *labs,
                  const i64 *Poff, double *Y) {
    for (i64 idx = 0; idx < nr; idx++) {
        const i64 i = rows[idx];
        for (i64 c = 0; c < k; c++) {
            const double x = DD[idx * k + c];
            z[c] += x;
            for (i64 l = 0; l < nl; l++) Y[(Poff[l] + labs[l * n + i]) * k + c] += x;
        }
    }
}

/* vcsops.py:189-213 vcs_post (one owner): new effective multipliers SN of moved rows at the current Y,
 * Z_R += d_i (SN v_new - stZ v_old), cnt_R += [SN>0] - [stZ>0], stZ = SN; batch-row order. */
void orc_vcs_post(i64 nr, const i64 *rows, i64 k, const double *V, const double *Vold, const double *d,
                  const i64 *lab, const double *Y, const i64 *ptr, const i32 *col, const double *sig, double *stZ,
                  const double *rq, double wv, double rho, double *Z, double *cnt) {
    for (i64 idx = 0; idx < nr; idx++) {
        const i64 i = rows[idx], Ri = lab[i];
        const double di = d[i];
        for (i64 e = ptr[i]; e < ptr[i + 1]; e++) {
            const i64 R = col[e];
            double sn;
            if (rho > 0.0 && di > 0.0) {
                double s = 0.0;
                for (i64 c = 0; c < k; c++) s += V[i * k + c] * Y[R * k + c];
                const double g = (R == Ri) ? di * (s - di) : di * s;
                const double p = sig[e] - rho * (wv * rq[R] / (di * di)) * g;
                sn = p > 0.0 ? p : 0.0;
            } else
                sn = sig[e];
            const double so = stZ[e];
            if (sn != 0.0 || so != 0.0)
                for (i64 c = 0; c < k; c++) Z[R * k + c] += di * (sn * V[i * k + c] - so * Vold[idx * k + c]);
            if (sn > 0.0) {
                if (!(so > 0.0)) cnt[R] += 1.0;
            } else if (so > 0.0)
                cnt[R] -= 1.0;
            stZ[e] = sn;
        }
    }
}

/* alm_vcs.py:378-415 pair_all (ne_split off) with a dense sigma: for every listed cluster Q of one level,
 * M[Q] = sum_R pp_QR Y_R, pdiag[Q] = pp_QQ, pp = max(0, sig - rho rq_Q rq_R w h) (rho = 0: pp = sig).
 * The reference is compiled with fastmath(reassoc, contract): this restatement sums in R order without FMA. */
void orc_pair_rows(i64 nitems, const i64 *items, i64 P, i64 k, const double *Y, const double *sig, const double *rq,
                   const double *dsq, double w, double rho, double *M, double *pdiag) {
#pragma omp parallel for schedule(dynamic, 4)
    for (i64 t = 0; t < nitems; t++) {
        const i64 Q = items[t];
        double acc[1024], pq = 0.0;
        for (i64 c = 0; c < k; c++) acc[c] = 0.0;
        for (i64 R = 0; R < P; R++) {
            double p;
            if (rho > 0.0) {
                double h = 0.0;
                for (i64 c = 0; c < k; c++) h += Y[Q * k + c] * Y[R * k + c];
                if (R == Q) h -= dsq[Q];
                p = sig[Q * P + R] - (rho * ((rq[Q] * rq[R]) * w)) * h;
                if (p < 0.0) p = 0.0;
            } else
                p = sig[Q * P + R];
            if (R == Q) pq = p;
            if (p != 0.0)
                for (i64 c = 0; c < k; c++) acc[c] += p * Y[R * k + c];
        }
        pdiag[Q] = pq;
        for (i64 c = 0; c < k; c++) M[Q * k + c] = acc[c];
    }
}

/* alm_vcs.py:417-428 kq_level with r = rq rq^T w: Kq = 2 rho (sum_{pp>0} r y2 + [pp_QQ>0] r_QQ y2_Q) */
void orc_kq(i64 P, const double *H, const double *sig, const double *rq, double w, const double *y2, double rho,
            double *out) {
    for (i64 Q = 0; Q < P; Q++) {
        double s = 0.0;
        for (i64 R = 0; R < P; R++) {
            const double r = (rq[Q] * rq[R]) * w;
            const double p = sig[Q * P + R] - rho * r * H[Q * P + R];
            if (p > 0.0) s += r * y2[R];
        }
        const double rQQ = (rq[Q] * rq[Q]) * w;
        const double pq = sig[Q * P + Q] - rho * rQQ * H[Q * P + Q];
        const double dg = pq > 0.0 ? rQQ * y2[Q] : 0.0;
        out[Q] = 2 * rho * (s + dg);
    }
}

/* alm_vcs.py:256-351 batch_step6 restricted to the production features (no neighbour/connectivity/pair cuts,
 * ne_split off) in the Jacobi-within-batch form: every batch row steps from the pre-batch V (read from V, written to
 * Vnew; rows of V not in the batch are left to the caller).  Per-row arithmetic follows the reference line by line:
 *   g = -(d_i/L)(z - d_i v_i) + sum_j w_ij v_j + sum_l d_i (M_Q - pdiag_Q d_i v_i) + GX - 1/2 sum_t pt q_t,
 *   kap = sum_l d_i^2 Kq_Q + KX + rt sum_{pt>0} |q_t|^2,  v <- normalize(g + (kap/2 + damp |g|) v),
 *   DD = d_i (v_new - v_old).  Triangle records are read in incidence order (IABC/LINC = TI[t], lam[t]). */
void orc_batch_step(i64 nr, const i64 *rows, i64 n, i64 k, const double *V, double *Vnew, const i64 *indptr,
                    const i64 *indices, const double *adata, const double *d, const double *z, double L, i64 nl,
                    const i64 *labs, const i64 *Poff, const double *Mall, const double *pdiag, const double *Kq,
                    const i64 *tptr, const i64 *tcodes, const i64 *TI, const double *lam, double rt, double damp,
                    int usevc, const double *GX, const double *KX, double *DD) {
#pragma omp parallel for schedule(dynamic, 16)
    for (i64 idx = 0; idx < nr; idx++) {
        const i64 i = rows[idx];
        const double di = d[i];
        const double *vi = V + i * k;
        double g[1024], q[1024];
        for (i64 c = 0; c < k; c++) g[c] = -(di / L) * (z[c] - di * vi[c]);
        for (i64 e = indptr[i]; e < indptr[i + 1]; e++) {
            const double w = adata[e];
            const double *vj = V + indices[e] * k;
            for (i64 c = 0; c < k; c++) g[c] += w * vj[c];
        }
        double kap = 0.0;
        for (i64 l = 0; l < nl; l++) {
            const i64 Q = Poff[l] + labs[l * n + i];
            const double *mq = Mall + Q * k;
            const double pd = pdiag[Q] * di;
            for (i64 c = 0; c < k; c++) g[c] += di * (mq[c] - pd * vi[c]);
            kap += di * di * Kq[Q];
        }
        if (usevc) {
            for (i64 c = 0; c < k; c++) g[c] += GX[idx * k + c];
            kap += KX[idx];
        }
        for (i64 e = tptr[i]; e < tptr[i + 1]; e++) {
            const i64 code = tcodes[e], t = code / 3, r = code % 3;
            const double *va = V + TI[3 * t] * k, *vb = V + TI[3 * t + 1] * k, *vc = V + TI[3 * t + 2] * k;
            double tau = 0.0, q2 = 0.0;
            for (i64 c = 0; c < k; c++) {
                const double a_ = va[c], b_ = vb[c], c_ = vc[c];
                tau += a_ * b_ + b_ * c_ - a_ * c_;
                q[c] = (r == 0) ? b_ - c_ : (r == 1) ? a_ + c_ : b_ - a_;
                q2 += q[c] * q[c];
            }
            const double pt = lam[t] - rt * (1.0 - tau);
            if (pt > 0.0) {
                for (i64 c = 0; c < k; c++) g[c] -= 0.5 * pt * q[c];
                kap += rt * q2;
            }
        }
        double gn = 0.0;
        for (i64 c = 0; c < k; c++) gn += g[c] * g[c];
        const double w = 0.5 * kap + damp * sqrt(gn);
        double nv = 0.0;
        for (i64 c = 0; c < k; c++) {
            q[c] = g[c] + w * vi[c];
            nv += q[c] * q[c];
        }
        double *vo = Vnew + i * k;
        if (nv <= 0.0) {
            for (i64 c = 0; c < k; c++) {
                DD[idx * k + c] = 0.0;
                vo[c] = vi[c];
            }
            continue;
        }
        nv = 1.0 / sqrt(nv);
        for (i64 c = 0; c < k; c++) {
            const double vn = q[c] * nv;
            vo[c] = vn;
            DD[idx * k + c] = di * (vn - vi[c]);
        }
    }
}

/* ---------------------------------------------------------------------------------------------- separation
 * Candidate enumeration of the two wedge families in generation order (centre j ascending, then arm pairs):
 *   family 0 (edge arms):   alm_vcs.py:554-565 _centre, 567-597 sep_hist / sep_collect,
 *   family 1 (one-edge-arm): alm_vcs.py:608-632 _centre1, 634-666 sep1_hist / sep1_collect.
 * Every violation vm > vtol is emitted (vm, min(a, c), j, max(a, c)); the histogram threshold, per-chunk caps and
 * collection of separate_ref / separate1_ref (alm_vcs.py:965-984) are applied by the Python side.  Top-k selections
 * sort by value descending with ties kept in input order (np.argsort is unstable: tied values are the only
 * documented difference). */
static double dot_rows(const double *V, i64 k, i64 a, i64 b) {
    double s = 0.0;
    for (i64 q = 0; q < k; q++) s += V[a * k + q] * V[b * k + q];
    return s;
}

typedef struct {
    i64 id;
    double x;
    i64 pos;
} arm_t;

static int cmp_desc(const void *A, const void *B) {
    const arm_t *a = (const arm_t *)A, *b = (const arm_t *)B;
    if (a->x > b->x) return -1;
    if (a->x < b->x) return 1;
    return (a->pos < b->pos) ? -1 : (a->pos > b->pos);
}

static int cmp_id(const void *A, const void *B) {
    const arm_t *a = (const arm_t *)A, *b = (const arm_t *)B;
    if (a->id != b->id) return (a->id < b->id) ? -1 : 1;
    return (a->pos < b->pos) ? -1 : (a->pos > b->pos);
}

/* _centre: neighbours i of j with X_ij > thresh (edge order); if more than maxh, the top maxh by X descending */
static i64 centre(i64 j, const i64 *indptr, const i64 *indices, const double *V, i64 k, double thresh, i64 maxh,
                  arm_t *H) {
    i64 m = 0;
    for (i64 e = indptr[j]; e < indptr[j + 1]; e++) {
        const i64 i = indices[e];
        double s = 0.0;
        for (i64 q = 0; q < k; q++) s += V[i * k + q] * V[j * k + q];
        if (s > thresh) {
            H[m].id = i;
            H[m].x = s;
            H[m].pos = m;
            m++;
        }
    }
    if (m > maxh) {
        qsort(H, m, sizeof(arm_t), cmp_desc);
        m = maxh;
    }
    return m;
}

static int isadj(const i64 *indptr, const i64 *indices, i64 j, i64 x) {
    i64 lo = indptr[j], hi = indptr[j + 1];
    while (lo < hi) {
        const i64 mid = (lo + hi) / 2;
        if (indices[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo < indptr[j + 1] && indices[lo] == x;
}

/* emits into (out_tri, out_val) up to cap entries; returns the total count (the caller re-runs with a bigger cap) */
i64 orc_sep_candidates(int family, i64 n, i64 k, const i64 *indptr, const i64 *indices, const double *V,
                       double thresh, i64 maxh, i64 maxk, i64 hub2, i64 cap2, double vtol, i64 cap, i64 *out_tri,
                       double *out_val) {
    i64 maxdeg = 0;
    for (i64 j = 0; j < n; j++)
        if (indptr[j + 1] - indptr[j] > maxdeg) maxdeg = indptr[j + 1] - indptr[j];
    arm_t *H = (arm_t *)malloc(sizeof(arm_t) * (maxdeg + 1));
    arm_t *Kc = (arm_t *)malloc(sizeof(arm_t) * (hub2 * cap2 + 1));
    i64 cnt = 0;
    for (i64 j = 0; j < n; j++) {
        const i64 dj = indptr[j + 1] - indptr[j];
        if (family == 0 && dj < 2) continue;
        if (family == 1 && dj < 1) continue;
        const i64 mh = centre(j, indptr, indices, V, k, thresh, maxh, H);
        if (family == 0) {
            for (i64 x = 0; x < mh; x++)
                for (i64 y = x + 1; y < mh; y++) {
                    const double s = dot_rows(V, k, H[x].id, H[y].id);
                    const double vm = H[x].x + H[y].x - s - 1.0;
                    if (vm > vtol) {
                        if (cnt < cap) {
                            const i64 a = H[x].id, c = H[y].id;
                            out_tri[3 * cnt] = a < c ? a : c;
                            out_tri[3 * cnt + 1] = j;
                            out_tri[3 * cnt + 2] = a < c ? c : a;
                            out_val[cnt] = vm;
                        }
                        cnt++;
                    }
                }
            continue;
        }
        /* _centre1: non-edge arms through the hub2 strongest arms, at most cap2 neighbours each */
        const i64 nh = mh < hub2 ? mh : hub2;
        i64 m = 0;
        for (i64 a = 0; a < nh; a++) {
            const i64 i2 = H[a].id, lo = indptr[i2];
            const i64 hi = (indptr[i2 + 1] < lo + cap2) ? indptr[i2 + 1] : lo + cap2;
            for (i64 e = lo; e < hi; e++) {
                const i64 c = indices[e];
                if (c == j || isadj(indptr, indices, j, c)) continue;
                double s = 0.0;
                for (i64 q = 0; q < k; q++) s += V[c * k + q] * V[j * k + q];
                if (s > thresh) {
                    Kc[m].id = c;
                    Kc[m].x = s;
                    Kc[m].pos = m;
                    m++;
                }
            }
        }
        if (m > 1) {
            qsort(Kc, m, sizeof(arm_t), cmp_id);
            i64 w = 1;
            for (i64 t = 1; t < m; t++)
                if (Kc[t].id != Kc[w - 1].id) Kc[w++] = Kc[t];
            m = w;
            for (i64 t = 0; t < m; t++) Kc[t].pos = t;
        }
        if (m > maxk) {
            qsort(Kc, m, sizeof(arm_t), cmp_desc);
            m = maxk;
        }
        if (m == 0 || mh == 0) continue;
        for (i64 x = 0; x < mh; x++)
            for (i64 y = 0; y < m; y++) {
                if (H[x].id == Kc[y].id) continue;
                const double s = dot_rows(V, k, H[x].id, Kc[y].id);
                const double vm = H[x].x + Kc[y].x - s - 1.0;
                if (vm > vtol) {
                    if (cnt < cap) {
                        const i64 a = H[x].id, c = Kc[y].id;
                        out_tri[3 * cnt] = a < c ? a : c;
                        out_tri[3 * cnt + 1] = j;
                        out_tri[3 * cnt + 2] = a < c ? c : a;
                        out_val[cnt] = vm;
                    }
                    cnt++;
                }
            }
    }
    free(H);
    free(Kc);
    return cnt;
}
