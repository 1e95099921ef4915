// pcg (src/pressure.rs:341-397) on one thread-block cluster, for fluid
// regions too large for the one-block kernel k_pcg.
//
// Same wavefront layout, vectors and per-cell f64 arithmetic as k_pcg: the
// MIC(0) factor (pressure.rs:442-513) and the two triangular sweeps
// (pressure.rs:517-570) walk the i+j+k levels in order, but every level is
// spread over all threads of the cluster (up to 16 CTAs on 16 SMs) and the
// levels are separated by the hardware cluster barrier (barrier.cluster with
// release/acquire), not a software grid barrier: no thread spins on memory.
// Values that other CTAs wrote during the solve are read through L2
// (ld.global.cg), so no stale L1 line is ever used.
//
// Dot products: the helpers of pressure.cuh. In exact mode the reference's
// 4096-cell chunks (pressure.rs:588-603) are folded one warp per chunk across
// the cluster and the chunk sums added in chunk order, bit-identical to k_pcg
// and to the reference; the default tree order (fixed 256-cell tiles) is the
// same as k_pcg's too, so both kernels give the same pressure bits.
#pragma once
#include "pressure.cuh"

namespace sdr {

constexpr int kClBS = 512;           // threads per CTA
constexpr int kClMaxCtas = 16;       // largest cluster (non-portable size)
constexpr int kClMaxLevelsSmem = 4096;


struct ClusterCtx {
    int rank, nctas;
    int gtid, gthreads;   // thread index and count over the cluster
    const int* lvs;       // level starts (shared memory, or global when many)
};

// build_mic0 (pressure.rs:442-513): forward level sweep over the cluster,
// the same per-cell arithmetic as pcg_build_mic0.
__device__ void cl_build_mic0(const PcgArgs& a, const ClusterCtx& c, int l0, int l1) {
    const double TAU = 0.97, SIGMA = 0.25;
    for (int L = l0; L < l1; ++L) {
        const int ls = c.lvs[L], le = c.lvs[L + 1];
        for (int ps = ls + c.gtid; ps < le; ps += c.gthreads) {
            const int* nb = a.nbr + (size_t)ps * 6;
            double axi = 0, pxi = 0, axi_y = 0, axi_z = 0;
            double ayj = 0, pyj = 0, ayj_x = 0, ayj_z = 0;
            double azk = 0, pzk = 0, azk_x = 0, azk_y = 0;
            int mm = nb[NB_MX];
            if (mm >= 0) {
                int mk = a.nmask[mm];
                axi = -1.0;
                pxi = __ldcg(a.precon + mm);
                axi_y = (mk >> NB_PY & 1) ? -1.0 : 0.0;
                axi_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            mm = nb[NB_MY];
            if (mm >= 0) {
                int mk = a.nmask[mm];
                ayj = -1.0;
                pyj = __ldcg(a.precon + mm);
                ayj_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                ayj_z = (mk >> NB_PZ & 1) ? -1.0 : 0.0;
            }
            mm = nb[NB_MZ];
            if (mm >= 0) {
                int mk = a.nmask[mm];
                azk = -1.0;
                pzk = __ldcg(a.precon + mm);
                azk_x = (mk >> NB_PX & 1) ? -1.0 : 0.0;
                azk_y = (mk >> NB_PY & 1) ? -1.0 : 0.0;
            }
            double tx = dmul(axi, pxi), ty = dmul(ayj, pyj), tz = dmul(azk, pzk);
            double diag = (double)a.diag[ps];
            double mx = dmul(dmul(dmul(axi, dadd(axi_y, axi_z)), pxi), pxi);
            double my = dmul(dmul(dmul(ayj, dadd(ayj_x, ayj_z)), pyj), pyj);
            double mz = dmul(dmul(dmul(azk, dadd(azk_x, azk_y)), pzk), pzk);
            double e = dsub(dsub(dsub(dsub(diag, dmul(tx, tx)), dmul(ty, ty)), dmul(tz, tz)),
                            dmul(TAU, dadd(dadd(mx, my), mz)));
            if (e < dmul(SIGMA, diag)) e = diag;
            a.precon[ps] = e > 0.0 ? ddiv(1.0, __dsqrt_rn(e)) : 0.0;
        }
        cluster_sync_all();
    }
}

// apply_mic0 (pressure.rs:517-570): forward L q = r, backward L^T z = q, and
// the z*r products of the following dot into `prod` (cell order for the
// reference dots, wavefront order for the tree dots). A thread's first cell of
// the next level (its neighbour indices, operand and factor, none of which the
// sweep writes) is loaded before the level barrier, so after the barrier only
// the neighbours' sweep values are on the critical path; further cells of wide
// levels load inline.
__device__ void cl_apply_mic0(const PcgArgs& a, const ClusterCtx& c, const double* r, double* z, int l0, int l1) {
    const int G = c.gthreads;
    // ---------------- forward
    int ps = c.lvs[l0] + c.gtid, le = c.lvs[l0 + 1];
    int mx = -1, my = -1, mz = -1;
    double rv = 0.0, pc = 0.0;
    if (ps < le) {
        const int* nb = a.nbr + (size_t)ps * 6;
        mx = nb[NB_MX]; my = nb[NB_MY]; mz = nb[NB_MZ];
        rv = __ldcg(r + ps);
        pc = __ldcg(a.precon + ps);
    }
    for (int L = l0; L < l1; ++L) {
        const int nps = le + c.gtid, nle = L + 1 < l1 ? c.lvs[L + 2] : le;
        int nmx = -1, nmy = -1, nmz = -1;
        double nrv = 0.0, npc = 0.0;
        if (nps < nle) {
            const int* nb = a.nbr + (size_t)nps * 6;
            nmx = nb[NB_MX]; nmy = nb[NB_MY]; nmz = nb[NB_MZ];
            nrv = __ldcg(r + nps);
            npc = __ldcg(a.precon + nps);
        }
        if (ps < le) {
            double vx = mx >= 0 ? __ldcg(a.pq + mx) : 0.0;
            double vy = my >= 0 ? __ldcg(a.pq + my) : 0.0;
            double vz = mz >= 0 ? __ldcg(a.pq + mz) : 0.0;
            double t = rv;
            if (mx >= 0) t = dadd(t, vx);
            if (my >= 0) t = dadd(t, vy);
            if (mz >= 0) t = dadd(t, vz);
            double qv = dmul(t, pc);
            a.q[ps] = qv;
            a.pq[ps] = dmul(pc, qv);
            for (int p2 = ps + G; p2 < le; p2 += G) {
                const int* nb = a.nbr + (size_t)p2 * 6;
                const int x = nb[NB_MX], y = nb[NB_MY], zz = nb[NB_MZ];
                double t2 = __ldcg(r + p2), pc2 = __ldcg(a.precon + p2);
                double wx = x >= 0 ? __ldcg(a.pq + x) : 0.0;
                double wy = y >= 0 ? __ldcg(a.pq + y) : 0.0;
                double wz = zz >= 0 ? __ldcg(a.pq + zz) : 0.0;
                if (x >= 0) t2 = dadd(t2, wx);
                if (y >= 0) t2 = dadd(t2, wy);
                if (zz >= 0) t2 = dadd(t2, wz);
                double q2 = dmul(t2, pc2);
                a.q[p2] = q2;
                a.pq[p2] = dmul(pc2, q2);
            }
        }
        cluster_sync_all();
        ps = nps; le = nle;
        mx = nmx; my = nmy; mz = nmz;
        rv = nrv; pc = npc;
    }
    // ---------------- backward
    int ls = c.lvs[l1 - 1];
    ps = ls + c.gtid;
    le = c.lvs[l1];
    int px = -1, py = -1, pz = -1;
    double qv = 0.0, rr = 0.0;
    pc = 0.0;
    if (ps < le) {
        const int* nb = a.nbr + (size_t)ps * 6;
        px = nb[NB_PX]; py = nb[NB_PY]; pz = nb[NB_PZ];
        qv = __ldcg(a.q + ps);
        rr = __ldcg(r + ps);
        pc = __ldcg(a.precon + ps);
    }
    for (int L = l1 - 1; L >= l0; --L) {
        const int nls = L - 1 >= l0 ? c.lvs[L - 1] : ls;
        const int nps = nls + c.gtid, nle = ls;
        int npx = -1, npy = -1, npz = -1;
        double nqv = 0.0, nrr = 0.0, npc = 0.0;
        if (nps < nle) {
            const int* nb = a.nbr + (size_t)nps * 6;
            npx = nb[NB_PX]; npy = nb[NB_PY]; npz = nb[NB_PZ];
            nqv = __ldcg(a.q + nps);
            nrr = __ldcg(r + nps);
            npc = __ldcg(a.precon + nps);
        }
        if (ps < le) {
            double vx = px >= 0 ? __ldcg(z + px) : 0.0;
            double vy = py >= 0 ? __ldcg(z + py) : 0.0;
            double vz = pz >= 0 ? __ldcg(z + pz) : 0.0;
            double t = qv;
            if (px >= 0) t = dadd(t, dmul(pc, vx));
            if (py >= 0) t = dadd(t, dmul(pc, vy));
            if (pz >= 0) t = dadd(t, dmul(pc, vz));
            double zv = dmul(t, pc);
            z[ps] = zv;
            a.prod[a.exact_dots ? a.cinv[ps] : ps] = dmul(zv, rr);
            for (int p2 = ps + G; p2 < le; p2 += G) {
                const int* nb = a.nbr + (size_t)p2 * 6;
                const int x = nb[NB_PX], y = nb[NB_PY], zz = nb[NB_PZ];
                double pc2 = __ldcg(a.precon + p2);
                double t2 = __ldcg(a.q + p2);
                double wx = x >= 0 ? __ldcg(z + x) : 0.0;
                double wy = y >= 0 ? __ldcg(z + y) : 0.0;
                double wz = zz >= 0 ? __ldcg(z + zz) : 0.0;
                if (x >= 0) t2 = dadd(t2, dmul(pc2, wx));
                if (y >= 0) t2 = dadd(t2, dmul(pc2, wy));
                if (zz >= 0) t2 = dadd(t2, dmul(pc2, wz));
                double z2 = dmul(t2, pc2);
                z[p2] = z2;
                a.prod[a.exact_dots ? a.cinv[p2] : p2] = dmul(z2, __ldcg(r + p2));
            }
        }
        cluster_sync_all();
        ls = nls;
        ps = nps; le = nle;
        px = npx; py = npy; pz = npz;
        qv = nqv; rr = nrr; pc = npc;
    }
}

// The solve. Launched as exactly one cluster (gridDim = cluster size).
// `slots` holds 2 x kClMaxCtas doubles of scratch for the CTA partials.
__global__ void __launch_bounds__(kClBS, 1) k_pcg_cluster(PcgArgs a) {
    __shared__ int s_lvs[kClMaxLevelsSmem + 1];
    __shared__ double sh[40];
    __shared__ int s_l0, s_l1;
    ClusterCtx c;
    c.rank = (int)cluster_rank();
    c.nctas = (int)cluster_size();
    c.gtid = c.rank * kClBS + (int)threadIdx.x;
    c.gthreads = c.nctas * kClBS;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (a.nlevels <= kClMaxLevelsSmem) {
        for (int L = tid; L <= a.nlevels; L += nt) s_lvs[L] = a.level_start[L];
        c.lvs = s_lvs;
    } else {
        c.lvs = a.level_start;
    }
    if (tid == 0) {
        s_l0 = a.nlevels;
        s_l1 = 0;
    }
    __syncthreads();
    for (int L = tid; L < a.nlevels; L += nt) {
        if (c.lvs[L + 1] > c.lvs[L]) {
            atomicMin(&s_l0, L);
            atomicMax(&s_l1, L + 1);
        }
    }
    __syncthreads();
    const int l0 = s_l0, l1 = s_l1;
    const uint32_t nf = *a.nf;
    const int G = c.gthreads, gt = c.gtid;

    PcgCl pc = pcg_cl();
    const uint32_t ntile = (nf + kTile - 1) / kTile;
    const int lane = tid & 31;
    double mx = 0.0;
    for (uint32_t i = gt; i < nf; i += G) mx = fmax(mx, fabs(a.b[i]));
    double residual = pcg_cl_max<kClBS>(pc, a, mx, sh);
    int iters = 0;
    if (residual > a.tol) {
        cl_build_mic0(a, c, l0, l1);
        for (uint32_t i = gt; i < nf; i += G) {
            a.r[i] = a.b[i];
            a.p[i] = 0.0;
        }
        cluster_sync_all();
        cl_apply_mic0(a, c, a.r, a.z, l0, l1);
        double sigma = pcg_dot_prod(a, pc, nf, sh);  // dot(z, r)
        for (uint32_t i = gt; i < nf; i += G) a.s[i] = __ldcg(a.z + i);
        cluster_sync_all();  // s complete before the matvec reads neighbours
        for (int it = 0; it < a.max_iters; ++it) {
            iters = it + 1;
            // apply_a (pressure.rs:400-439) and s*As, by tiles of the tree dot
            for (uint32_t t = (uint32_t)pc.gw; t < ntile; t += (uint32_t)pc.nw) {
                double acc = 0.0;
                for (int u = 0; u < kTile / 32; ++u) {
                    const uint32_t i = t * kTile + lane + 32u * u;
                    if (i >= nf) break;
                    const int2* nb2 = reinterpret_cast<const int2*>(a.nbr + (size_t)i * 6);
                    int2 x0 = nb2[0], x1 = nb2[1], x2 = nb2[2];
                    int nbv[6] = {x0.x, x0.y, x1.x, x1.y, x2.x, x2.y};
                    double sv = __ldcg(a.s + i);
                    double nsv[6];
#pragma unroll
                    for (int d = 0; d < 6; ++d) nsv[d] = nbv[d] >= 0 ? __ldcg(a.s + nbv[d]) : 0.0;
                    double v = dmul((double)a.diag[i], sv);
                    if (nbv[NB_PX] >= 0) v = dsub(v, nsv[NB_PX]);
                    if (nbv[NB_MX] >= 0) v = dsub(v, nsv[NB_MX]);
                    if (nbv[NB_PY] >= 0) v = dsub(v, nsv[NB_PY]);
                    if (nbv[NB_MY] >= 0) v = dsub(v, nsv[NB_MY]);
                    if (nbv[NB_PZ] >= 0) v = dsub(v, nsv[NB_PZ]);
                    if (nbv[NB_MZ] >= 0) v = dsub(v, nsv[NB_MZ]);
                    a.as[i] = v;
                    if (a.exact_dots) a.prod[a.cinv[i]] = dmul(sv, v);
                    else acc = dadd(acc, dmul(sv, v));
                }
                if (!a.exact_dots) {
                    acc = warp_tree_sum(acc);
                    if (lane == 0) a.tpart[t] = acc;
                }
            }
            double denom;  // dot(s, As)
            if (a.exact_dots) {
                denom = pcg_exact_dot(a, pc, sh);
            } else {
                cluster_sync_all();
                denom = pcg_tile_total(a, ntile);
            }
            if (fabs(denom) < 1e-30) break;
            double alpha = ddiv(sigma, denom);
            double mr = 0.0;
            for (uint32_t i = gt; i < nf; i += G) {
                a.p[i] = dadd(a.p[i], dmul(alpha, __ldcg(a.s + i)));
                double rv = dsub(a.r[i], dmul(alpha, __ldcg(a.as + i)));
                a.r[i] = rv;
                mr = fmax(mr, fabs(rv));
            }
            residual = pcg_cl_max<kClBS>(pc, a, mr, sh);  // also orders r before the sweeps
            if (residual <= a.tol) break;
            cl_apply_mic0(a, c, a.r, a.z, l0, l1);
            double sigma_new = pcg_dot_prod(a, pc, nf, sh);  // dot(z, r)
            double beta = ddiv(sigma_new, sigma);
            for (uint32_t i = gt; i < nf; i += G) a.s[i] = dadd(__ldcg(a.z + i), dmul(beta, a.s[i]));
            cluster_sync_all();  // s complete before the next matvec reads neighbours
            sigma = sigma_new;
        }
        for (uint32_t i = gt; i < nf; i += G) a.p_dense[a.lv_cell[i]] = a.p[i];
    }
    if (c.rank == 0 && tid == 0) {
        *a.out_iters = iters;
        *a.out_residual = residual;
    }
    cluster_sync_all();  // no CTA exits while another may still read its slots
}

}  // namespace sdr
