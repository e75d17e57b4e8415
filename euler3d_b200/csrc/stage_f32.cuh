// FP32_FLUX stage kernel: fluxes, face states and the time step in single precision; the
// conservative state W0, the residual sums, the Runge-Kutta update and every reduction in double.
//
// Same face-tile scheme as tile_kernel (stage.cuh): one block per tile of kTileCells Morton-ordered
// cells, bulk copies of the tile's contiguous data plus cp.async gathers of its halo onto one
// mbarrier, each face evaluated once, each cell summing its faces' F*S in ascending reference face
// id (deterministic).  Cell records are 32 bytes (two float4), face records 24 bytes, so a tile's
// staging is about half the double-precision one and eight blocks fit on an SM.
#pragma once
#include "stage.cuh"

namespace e3d {

struct PrimF {
    float rho, u, v, w, p, H, s, r;  // s = sqrt(rho), r = rsqrt(gamma p rho)
};

__device__ __forceinline__ float rcp_f(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rsqrt_f(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Cell record of a double-precision state (written by the update and by the state loader).
__device__ __forceinline__ void make_rec32(float4 *dst, double rho, double u, double v, double w, double p, double H,
                                           double g) {
    const float fr = (float)rho, fp = (float)p;
    __stcs(dst, make_float4(fr, (float)u, (float)v, (float)w));  // streaming stores, as store_prim_cs
    __stcs(dst + 1, make_float4(fp, (float)H, fr * rsqrt_f(fr), rsqrt_f((float)g * fp * fr)));
}

// Roe flux with Harten's fix (Solver::Roe, src/solver/ConvectiveFluxesSchemes.cpp:10-165) in single
// precision, written as F = (F_L + F_R - sum_k a_k r_k) / 2 like roe_fast.  Built without
// multiply-add contraction: it fuses where the source writes fmaf(), so the rounding is fixed by
// the source in every kernel variant.
__device__ __forceinline__ void roe_f32(const PrimF &L, const PrimF &R, float nx, float ny, float nz, float g,
                                        float F[5]) {
    const float inv = rcp_f(L.s + R.s);
    const float wl = L.s * inv, wr = R.s * inv;
    const float ut = fmaf(L.u, wl, R.u * wr), vt = fmaf(L.v, wl, R.v * wr), wt = fmaf(L.w, wl, R.w * wr);
    const float ht = fmaf(L.H, wl, R.H * wr);
    const float rt = L.s * R.s;
    const float q2t = fmaf(ut, ut, fmaf(vt, vt, wt * wt));
    const float c2 = (g - 1.0f) * fmaf(-0.5f, q2t, ht);
    const float rc = rsqrt_f(c2);
    const float ct = c2 * rc, ic2 = rc * rc;
    const float Vt = fmaf(ut, nx, fmaf(vt, ny, wt * nz));
    const float Vl = fmaf(L.u, nx, fmaf(L.v, ny, L.w * nz));
    const float Vr = fmaf(R.u, nx, fmaf(R.v, ny, R.w * nz));
    const float drho = R.rho - L.rho, dp = R.p - L.p, dV = Vr - Vl;
    const float du = R.u - L.u, dv = R.v - L.v, dw = R.w - L.w;
    const float delta = (1.0f / 15.0f) * (g * L.p * L.r);
    float lam1 = fabsf(Vt - ct), lam5 = fabsf(Vt + ct);
    if (!(lam1 > delta) || !(lam5 > delta)) {
        const float h = 7.5f * (L.rho * L.r);
        if (!(lam1 > delta)) lam1 = fmaf(lam1, lam1, delta * delta) * h;
        if (!(lam5 > delta)) lam5 = fmaf(lam5, lam5, delta * delta) * h;
    }
    const float rcdv = rt * ct * dV;
    const float a1 = 0.5f * lam1 * (dp - rcdv) * ic2;
    const float a5 = 0.5f * lam5 * (dp + rcdv) * ic2;
    const float aV = fabsf(Vt);
    const float a2 = aV * fmaf(-dp, ic2, drho);
    const float a3 = aV * rt;
    const float a15 = a1 + a5, d51 = (a5 - a1) * ct, asum = a15 + a2;
    const float mL = L.rho * Vl, mR = R.rho * Vr, ps = L.p + R.p;
    F[0] = 0.5f * (mL + mR - asum);
    F[1] = 0.5f * (fmaf(mL, L.u, fmaf(mR, R.u, ps * nx)) - fmaf(asum, ut, fmaf(d51, nx, a3 * fmaf(-dV, nx, du))));
    F[2] = 0.5f * (fmaf(mL, L.v, fmaf(mR, R.v, ps * ny)) - fmaf(asum, vt, fmaf(d51, ny, a3 * fmaf(-dV, ny, dv))));
    F[3] = 0.5f * (fmaf(mL, L.w, fmaf(mR, R.w, ps * nz)) - fmaf(asum, wt, fmaf(d51, nz, a3 * fmaf(-dV, nz, dw))));
    F[4] = 0.5f * (fmaf(mL, L.H, mR * R.H) -
                   fmaf(a15, ht, fmaf(d51, Vt, fmaf(a2, 0.5f * q2t, a3 * fmaf(-Vt, dV, fmaf(ut, du, fmaf(vt, dv, wt * dw)))))));
}

// AUSM (Liou & Steffen 1993) in single precision; c = gamma p r, M = V rho r.
__device__ __forceinline__ void ausm_f32(const PrimF &L, const PrimF &R, float nx, float ny, float nz, float g,
                                         float F[5]) {
    const float cl = g * L.p * L.r, cr = g * R.p * R.r;
    const float Vl = fmaf(L.u, nx, fmaf(L.v, ny, L.w * nz)), Vr = fmaf(R.u, nx, fmaf(R.v, ny, R.w * nz));
    const float Ml = Vl * (L.rho * L.r), Mr = Vr * (R.rho * R.r);
    float mp, pp, mm, pm;
    if (fabsf(Ml) <= 1.0f) {
        mp = 0.25f * (Ml + 1.0f) * (Ml + 1.0f);
        pp = mp * (2.0f - Ml);
    } else {
        mp = 0.5f * (Ml + fabsf(Ml));
        pp = Ml > 0.0f ? 1.0f : 0.0f;
    }
    if (fabsf(Mr) <= 1.0f) {
        mm = -0.25f * (Mr - 1.0f) * (Mr - 1.0f);
        pm = -mm * (2.0f + Mr);
    } else {
        mm = 0.5f * (Mr - fabsf(Mr));
        pm = Mr < 0.0f ? 1.0f : 0.0f;
    }
    const float mi = mp + mm, pi = fmaf(pp, L.p, pm * R.p);
    const float al = fmaxf(mi, 0.0f) * (L.rho * cl), ar = fminf(mi, 0.0f) * (R.rho * cr);
    F[0] = al + ar;
    F[1] = fmaf(al, L.u, fmaf(ar, R.u, pi * nx));
    F[2] = fmaf(al, L.v, fmaf(ar, R.v, pi * ny));
    F[3] = fmaf(al, L.w, fmaf(ar, R.w, pi * nz));
    F[4] = fmaf(al, L.H, ar * R.H);
}

__device__ __forceinline__ PrimF prim32(const float4 *st, int i) {
    const float4 a = st[2 * i], b = st[2 * i + 1];
    return PrimF{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
}

// Shared memory: st[LC] 32-byte records | rec[FC] | ct[MC][T] | mbarrier.  The five float F*S of
// face j are written over its 24-byte record (fs[6 j + k]), which only the thread evaluating the
// face reads.  W0 and the cell geometry stay in global memory (prefetched into L2 when the tile
// starts, read into registers before the flux phase ends), as in tile_body.
struct Tile32 {
    float4 *st;
    FaceRec32 *rec;
    unsigned short *ct;
};

__host__ __device__ __forceinline__ size_t tile32_buf_bytes(int LC, int FC, int MC) {
    return (size_t)LC * 32 + ((24u * (size_t)FC + 15) & ~(size_t)15) + (size_t)MC * kTileCells * 2;
}

__device__ __forceinline__ Tile32 tile32_at(unsigned char *base, int LC, int FC) {
    Tile32 b;
    b.st = reinterpret_cast<float4 *>(base);
    b.rec = reinterpret_cast<FaceRec32 *>(base + (size_t)LC * 32);
    b.ct = reinterpret_cast<unsigned short *>(base + (size_t)LC * 32 + round16(24u * FC));
    return b;
}

inline size_t tile32_smem_bytes(int smem_cells, int smem_faces, int max_contrib) {
    const size_t b = (tile32_buf_bytes(smem_cells, smem_faces, max_contrib) + 15) & ~(size_t)15;
    return b + 16;
}

// One flux per tile face, threads tid, tid + nt, ...; F*S of face j replaces record j.
__device__ __forceinline__ void tile_fluxes_f32(const StageArgs &a, const Tile32 &b, int nf, int c0, int tid, int nt) {
    const float gf = (float)a.gamma;
    float *fs = reinterpret_cast<float *>(b.rec);
    for (int j = tid; j < nf; j += nt) {
        const FaceRec32 fr = b.rec[j];
        const int l = fr.code & ((1 << kTileLocalBits) - 1);
        const int r = (fr.code >> kTileLocalBits) & ((1 << kTileLocalBits) - 1);
        const int tag = fr.code >> (2 * kTileLocalBits);
        const PrimF L = prim32(b.st, l);
        float F[5];
        if (tag == TAG_LEFT) {
            if (a.scheme == 1) ausm_f32(L, prim32(b.st, r), fr.nx, fr.ny, fr.nz, gf, F);
            else roe_f32(L, prim32(b.st, r), fr.nx, fr.ny, fr.nz, gf, F);
        } else {  // ghost cells are kept in double; their update uses the double boundary code
            const Prim Ld{L.rho, L.u, L.v, L.w, L.p, L.H};
            const double4 fg = make_double4(fr.nx, fr.ny, fr.nz, fr.S);
            double Fd[5];
            Prim gs;
            if (boundary_face(a, tag, a.ghost + 8 * (size_t)fr.ghost, c0 + l, Ld, fg, Fd, gs)) {
                const PrimF G{(float)gs.rho, (float)gs.u, (float)gs.v, (float)gs.w, (float)gs.p, (float)gs.H, L.s, L.r};
                if (a.scheme == 1) ausm_f32(L, G, fr.nx, fr.ny, fr.nz, gf, F);
                else roe_f32(L, G, fr.nx, fr.ny, fr.nz, gf, F);
            } else {
#pragma unroll
                for (int k = 0; k < 5; k++) F[k] = (float)Fd[k];
            }
        }
        // the record is in registers; keep the compiler from moving its loads past the overwrite
        asm volatile("" ::: "memory");
#pragma unroll
        for (int k = 0; k < 5; k++) fs[6 * j + k] = F[k] * fr.S;
    }
}

// The owner's W0 and geometry (global memory, prefetched into L2 when the tile started).
__device__ __forceinline__ void tile_load_cell_f32(const StageArgs &a, int c, double W0[5], float4 &cg) {
#pragma unroll
    for (int k = 0; k < 5; k++) W0[k] = __ldcs(a.w0 + (size_t)k * a.w0_stride + c);  // read once: streaming
    cg = __ldcs(a.cgeo32 + c);
}

// Cell i of the tile: sum of its faces' F*S, time step and update; returns R_rho^2 on the last stage.
__device__ __forceinline__ double tile_update_f32(const StageArgs &a, const Tile32 &b, int c0, int i, const double W0[5],
                                                  const float4 &cg) {
    const int T = kTileCells, MC = a.max_contrib;
    const float gf = (float)a.gamma;
    const float *fs = reinterpret_cast<const float *>(b.rec);
    const PrimF me = prim32(b.st, i);
    double R[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    unsigned short e[6];
#pragma unroll
    for (int k = 0; k < 6; k++) e[k] = k < MC ? b.ct[k * T + i] : kNoContrib;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        if (e[k] == kNoContrib) break;
        const int j = e[k] >> 1;
        const double sg = (e[k] & 1) ? -1.0 : 1.0;  // fma by -/+1: the bits of R -/+ F*S (see tile_update)
#pragma unroll
        for (int q = 0; q < 5; q++) R[q] = fma(sg, (double)fs[6 * j + q], R[q]);
    }
    // time step in single precision (TimeStepMethod2, src/solver/TimeIntegration.cpp:8-40)
    const float snd = gf * me.p * me.r;
    const float lam = 0.5f * fmaf(fabsf(me.u) + snd, cg.x, fmaf(fabsf(me.v) + snd, cg.y, (fabsf(me.w) + snd) * cg.z));
    const int c = c0 + i;
    if (a.residual_only) {
        const int o = a.new2old[c];
#pragma unroll
        for (int k = 0; k < 5; k++) a.r_out[5 * (size_t)o + k] = R[k];
        a.dt_out[o] = (double)(a.cfl * cg.w / lam);
        return 0.0;
    }
    // W = W0 - alpha dt R / V in double (alpha dt / V = alpha cfl / lambda)
    const double coef = a.alpha * a.cfl * rcp_nr((double)lam);
    double W[5];
#pragma unroll
    for (int k = 0; k < 5; k++) W[k] = fma(-coef, R[k], W0[k]);
    const double ir = rcp_nr(W[0]);
    const double u = W[1] * ir, v = W[2] * ir, w = W[3] * ir;
    const double p = (a.gamma - 1.0) * fma(-0.5, fma(W[1], u, fma(W[2], v, W[3] * w)), W[4]);
    const double H = (W[4] + p) * ir;
    make_rec32(a.q32out + 2 * (size_t)c, W[0], u, v, w, p, H, a.gamma);
    if (!a.last_stage) return 0.0;
    // the conservative state carries over exactly in double
    const size_t sd = (size_t)a.w0_stride;
#pragma unroll
    for (int k = 0; k < 5; k++) __stcs(a.w0 + k * sd + c, W[k]);
    __stcs(a.ecell + c, W[4] * ir);
    return R[0] * R[0];
}

// Body shared by tile_kernel_f32 (one solver) and tile_batch_kernel_f32 (several solvers in one
// grid): `tile` is the solver's own tile index, `partial` where its RMS partial goes.
__device__ __forceinline__ void tile_body_f32(const StageArgs &a, int tile, double *partial, unsigned char *smem_raw) {
    const int LC = a.smem_cells, FC = a.smem_faces, MC = a.max_contrib, T = kTileCells;
    const Tile32 b = tile32_at(smem_raw, LC, FC);
    const size_t off = (tile32_buf_bytes(LC, FC, MC) + 15) & ~(size_t)15;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + off);
    const int c0 = tile * T;
    const int nloc = min(T, a.n_cells - c0);
    // independent loads first, as in tile_body
    const int *hrow = a.tile_halo + (size_t)tile * a.halo_stride;
    const int i0 = threadIdx.x, i1 = threadIdx.x + T;
    const int hx0 = i0 < a.halo_stride ? hrow[i0] : -1;
    const int hx1 = i1 < a.halo_stride ? hrow[i1] : -1;
    const int fp0 = a.tile_face_ptr[tile], fp1 = a.tile_face_ptr[tile + 1];
    const long long rec_off = a.tile_rec32_off[tile];
    const bool done = !a.residual_only && a.ctl->done;
    const int nf = fp1 - fp0;

    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (done) return;  // uniform across the block
    if (threadIdx.x == 0) {
        const uint32_t b_state = (uint32_t)nloc * 32u;
        const uint32_t b_rec = round16(24u * (uint32_t)nf);
        const uint32_t b_w0 = round16((uint32_t)nloc * 8u);
        const uint32_t b_cg = (uint32_t)nloc * 16u;
        const uint32_t b_ct = (uint32_t)MC * T * 2u;
        mbar_expect_tx(bar, b_state + b_rec + b_ct);
        bulk_g2s(b.st, a.q32in + 2 * (size_t)c0, b_state, bar);
        const uint64_t once = l2_evict_first();
        bulk_g2s_hint(b.rec, a.tile_rec32 + rec_off, b_rec, bar, once);
        bulk_g2s_hint(b.ct, a.tile_contrib + (size_t)tile * MC * T, b_ct, bar, once);
        for (int k = 0; k < 5; k++) bulk_prefetch_l2(a.w0 + (size_t)k * a.w0_stride + c0, b_w0);
        bulk_prefetch_l2(a.cgeo32 + c0, b_cg);
    }
    auto gather = [&](int i, int h) {
        cp_async16(b.st + 2 * (nloc + i), a.q32in + 2 * (size_t)h);
        cp_async16(b.st + 2 * (nloc + i) + 1, a.q32in + 2 * (size_t)h + 1);
    };
    if (hx0 >= 0) gather(i0, hx0);
    if (hx1 >= 0) gather(i1, hx1);
    for (int i = threadIdx.x + 2 * T; i < a.halo_stride; i += T) {
        const int h = hrow[i];
        if (h >= 0) gather(i, h);
    }
    cp_async_wait_all();
    if (!tile_wait(a, bar, 0)) {
        tile_drain(bar, 0);
        return;
    }
    tile_fluxes_f32(a, b, nf, c0, threadIdx.x, kStageThreads);
    const int i = threadIdx.x;
    double W0[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    float4 cg = make_float4(0.f, 0.f, 0.f, 0.f);
    if (i < nloc) tile_load_cell_f32(a, c0 + i, W0, cg);  // latency overlaps the barrier's wait
    __syncthreads();
    double r2 = 0.0;
    if (i < nloc) r2 = tile_update_f32(a, b, c0, i, W0, cg);
    if (a.last_stage && !a.residual_only) block_sum_store(r2, partial);
}

template <int MINB>
__global__ void __launch_bounds__(kStageThreads, MINB) tile_kernel_f32(StageArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tile_body_f32(a, blockIdx.x, a.partials + blockIdx.x, smem_raw);
}

// Several solvers in one grid (see tile_batch_kernel).
template <int MINB>
__global__ void __launch_bounds__(kStageThreads, MINB) tile_batch_kernel_f32(BatchStage bs) {
    if ((int)blockIdx.x >= *bs.n_entries) return;
    __shared__ __align__(16) StageArgs sa;
    const int2 e = batch_stage_args(bs, &sa);
    if (sa.ctl->done) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tile_body_f32(sa, e.y, sa.partials + e.y, smem_raw);
}

}  // namespace e3d
