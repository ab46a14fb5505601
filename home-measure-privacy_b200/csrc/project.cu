// Projection of Gaussians into views, forward and backward.
//
// Forward: one thread per Gaussian reads its parameters once from the plane-major SoA
// (coalesced 128-byte rows per warp and plane) and projects it into every view of the
// batch, writing the pair's splat record, tile rectangle and depth key: PREPROCESS
// (trainer/gpu.js:64-88) plus the per-splat part of BIN (:626-635), with SH colour.
//
// Backward: one thread per Gaussian chains the screen gradients of every view
// (colour, opacity logit, u, v, conic) through the projection analytically; the
// reference does this by central differences of projectShape (SHAPE,
// trainer/gpu.js:297-328).  It writes all parameter planes once (no atomics).
#include "internal.h"

namespace gs {

// Approximate PTX instructions for the conservative tile spans (their slack covers the
// ~1e-6 relative error); the records themselves use exact rounding.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <int DEG>
__global__ void __launch_bounds__(128) project_fwd_kernel(ProjectArgs a) {
    constexpr int NK = (DEG + 1) * (DEG + 1) - 1;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_pad) return;
    const bool real = i < a.n;
    const int np = a.n_pad;
    float mean[3], ls[3], q[4], ol = 0.f, dc[3];
    if (real) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            mean[k] = __ldg(a.params + (0 + k) * np + i);
            ls[k] = __ldg(a.params + (3 + k) * np + i);
            dc[k] = __ldg(a.params + (11 + k) * np + i);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) q[k] = __ldg(a.params + (6 + k) * np + i);
        ol = __ldg(a.params + 10 * np + i);
    }
    float Sig[9];
    bool finite = false;
    float opacity = 0.f;
    if (real) {
        world_cov_exact(ls, q, Sig);
        opacity = xdiv(1.0f, xadd(1.0f, spec_expf(-ol)));
        finite = isfinite(mean[0]) && isfinite(mean[1]) && isfinite(mean[2]);
#pragma unroll
        for (int k = 0; k < 9; k++) finite = finite && isfinite(Sig[k]);
    }
    // Culling bound of the tile spans: alpha >= alpha_min needs the conic's quadratic
    // form <= 2 ln(opacity / alpha_min); the slack keeps the spans conservative against
    // the approximate arithmetic below and the raster's own rounding.
    const float thr_g = opacity > 0.f ? 2.0f * (__logf(opacity) - __logf(a.alpha_min)) + 1e-3f : -1.0f;
    unsigned int my_visible = 0, ok_views = 0;
    unsigned long long ok_mask = 0ull;  // views the Gaussian projects into (SH colour below)
    for (int s = 0; s < a.num_views; s++) {
        const ViewDesc& vw = a.views[a.view_first + s];
        const size_t pair = (size_t)(a.pair_slot_first + s) * np + i;
        Projected p;
        p.ok = false;
        if (finite) p = project_exact(vw, mean, Sig, a.near_plane, a.dilation);
        int x0 = 0, x1 = 0, y0 = 0, y1 = 0;
        if (p.ok && isfinite(p.u) && isfinite(p.v) && isfinite(p.radius))
            tile_rect(p.u, p.v, p.radius, vw.tiles_x, vw.tiles_y, a.rect_mode, vw.tile, x0, x1, y0, y1);
        else
            p.ok = false;
        uint32_t count = (p.ok && x1 > x0 && y1 > y0) ? (uint32_t)((x1 - x0) * (y1 - y0)) : 0u;
        uint32_t sp[GS_SPAN_ROWS / 2] = {};
        // Conic elongation kappa = A C / (A C - B^2): above 256 the ellipse arithmetic below
        // is not trusted (its rounding grows with kappa) and the whole rectangle is kept.
        const float kap_ac = p.a * p.c;
        const float kappa = p.ok ? kap_ac / fmaxf(kap_ac - p.b * p.b, kap_ac * 1e-12f + 1e-30f) : 0.f;
        if (count && a.tile_cull) {
            if (y1 - y0 <= GS_SPAN_ROWS && x1 - x0 < 256 && kappa <= 256.f) {
                // Per rectangle row, the tiles the ellipse A dx^2 + 2B dx dy + C dy^2 <= thr
                // reaches inside the row's pixel band (and the |d| <= r square, and the
                // image): the band's x-extent of the ellipse is contiguous, its right edge
                // concave and its left edge convex in dy, so each extreme sits at its
                // stationary point dy* = -/+ B sqrt(thr / (det C)) clamped to the band.
                const float thr = thr_g * (1.0f + kappa * 1.52587890625e-05f);  // rounding of the form grows with kappa
                const float A = p.a, B = p.b, C = p.c;
                const float det = fmaxf(A * C - B * B, 1e-30f);
                const float idet = rcp_approx(det);
                const float tp = fmaxf(thr, 0.f);
                const float ymax = sqrt_approx(tp * A * idet);
                const float ystat = B * sqrt_approx(tp * idet * rcp_approx(C));
                const float iA = rcp_approx(A);
                const float H1 = (float)vw.height - 0.5f, W1 = (float)vw.width - 0.5f;
                const float xlo_lim = fmaxf(p.u - p.radius, 0.5f), xhi_lim = fminf(p.u + p.radius, W1);
                const float slack = 1e-3f * (1.0f + p.radius);
                const int T = vw.tile;
                const float Tm = (float)T - 0.5f, iT = 1.0f / (float)T;
                count = 0;
#pragma unroll
                for (int r = 0; r < GS_SPAN_ROWS; r++) {
                    const int ty = y0 + r;
                    if (ty >= y1) break;
                    float yl = fmaxf(fmaxf((float)(ty * T) + 0.5f, p.v - p.radius), p.v - ymax) - p.v;
                    float yh = fminf(fminf(fminf((float)(ty * T) + Tm, H1), p.v + p.radius), p.v + ymax) - p.v;
                    int xs = 0, xe = 0;
                    if (thr > 0.f && yl <= yh) {
                        const float dr = fminf(fmaxf(-ystat, yl), yh);   // right edge maximiser
                        const float dl = fminf(fmaxf(ystat, yl), yh);    // left edge minimiser
                        const float sr = sqrt_approx(fmaxf(A * thr - det * dr * dr, 0.f));
                        const float sl = sqrt_approx(fmaxf(A * thr - det * dl * dl, 0.f));
                        const float xhi = fminf(p.u + (-B * dr + sr) * iA + slack, xhi_lim);
                        const float xlo = fmaxf(p.u + (-B * dl - sl) * iA - slack, xlo_lim);
                        if (xlo <= xhi) {
                            // Tile tx holds pixel centres [T tx + 0.5, T tx + T - 0.5].
                            xs = max(x0, __float2int_ru((xlo - Tm) * iT));
                            xe = min(x1, __float2int_rd((xhi - 0.5f) * iT) + 1);
                            if (xe < xs) xe = xs;
                        }
                    }
                    if (xe > xs) {
                        sp[r >> 1] |= ((uint32_t)(xs - x0) | ((uint32_t)(xe - x0) << 8)) << (16 * (r & 1));
                        count += (uint32_t)(xe - xs);
                    }
                }
            } else {
                count |= GS_PCOUNT_RECT;
            }
        } else if (count) {
            count |= GS_PCOUNT_RECT;
        }
        const bool covers = (count & ~GS_PCOUNT_RECT) != 0u;
        if (DEG == 0) a.rgb[pair] = p.ok ? make_float4(dc[0], dc[1], dc[2], 1.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
        if (p.ok) ok_mask |= 1ull << s;
        a.geo0[pair] = make_float4(p.ok ? p.u : 0.f, p.ok ? p.v : 0.f, p.ok ? p.a : 0.f, p.ok ? p.b : 0.f);
        a.geo1[pair] = make_float4(p.ok ? p.c : 0.f, p.ok ? opacity : 0.f, p.ok ? p.radius : 0.f,
                                   p.ok ? p.depth : 0.f);
        a.keys[pair] = covers ? __float_as_uint(p.depth) : GS_KEY_SENTINEL;
        a.pcount[pair] = covers ? count : 0u;
        if (covers) {
            uint4* er = reinterpret_cast<uint4*>(a.erec + pair);
            er[0] = make_uint4((uint32_t)(vw.tile_offset + y0 * vw.tiles_x + x0),
                               (uint32_t)vw.tiles_x | ((uint32_t)(x1 - x0) << 16) | (count & GS_PCOUNT_RECT), sp[4],
                               sp[5]);
            er[1] = make_uint4(sp[0], sp[1], sp[2], sp[3]);
        }
        my_visible += covers ? 1u : 0u;
        ok_views += p.ok ? 1u : 0u;
    }
    if (DEG > 0) {
        // SH colour per view, after the geometry: the 3 (K - 1) band coefficients are
        // loaded only now, so they do not hold registers through the projection.
        float sh[3][NK > 0 ? NK : 1];
        if (ok_mask) {
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int k = 0; k < NK; k++) sh[c][k] = __ldg(a.params + (14 + c * NK + k) * np + i);
        }
        for (int s = 0; s < a.num_views; s++) {
            const size_t pair = (size_t)(a.pair_slot_first + s) * np + i;
            float4 col = make_float4(0.f, 0.f, 0.f, 0.f);
            if (ok_mask >> s & 1ull) {
                const ViewDesc& vw = a.views[a.view_first + s];
                float r = dc[0], g = dc[1], b = dc[2];
                float dx = mean[0] - vw.campos[0], dy = mean[1] - vw.campos[1], dz = mean[2] - vw.campos[2];
                const float inv = rsqrtf(fmaxf(dx * dx + dy * dy + dz * dz, 1e-30f));
                dx *= inv; dy *= inv; dz *= inv;
                float Y[NK > 0 ? NK : 1];
                sh_basis(DEG, dx, dy, dz, Y);
#pragma unroll
                for (int k = 0; k < NK; k++) {
                    r += Y[k] * sh[0][k];
                    g += Y[k] * sh[1][k];
                    b += Y[k] * sh[2][k];
                }
                col = make_float4(r, g, b, 1.0f);
            }
            a.rgb[pair] = col;
        }
    }
    if (a.stats_cnt && ok_views) a.stats_cnt[i] += (float)ok_views;  // STATS count (trainer/gpu.js:494-496)
    if (a.visible) {
        // One atomic per warp.
        unsigned int sum = my_visible;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if ((threadIdx.x & 31) == 0 && sum) atomicAdd(a.visible, sum);
    }
}

void launch_project_fwd(const ProjectArgs& a, cudaStream_t s) {
    const int threads = 128;
    const int blocks = (a.n_pad + threads - 1) / threads;
    if (blocks == 0) return;
    switch (a.degree) {
        case 0: project_fwd_kernel<0><<<blocks, threads, 0, s>>>(a); break;
        case 1: project_fwd_kernel<1><<<blocks, threads, 0, s>>>(a); break;
        case 2: project_fwd_kernel<2><<<blocks, threads, 0, s>>>(a); break;
        default: project_fwd_kernel<3><<<blocks, threads, 0, s>>>(a); break;
    }
}

// ---------------------------------------------------------------------------------
// Backward.
// ---------------------------------------------------------------------------------
template <int DEG>
__global__ void __launch_bounds__(128, 4) project_bwd_kernel(ProjectBwdArgs a) {
    constexpr int NK = (DEG + 1) * (DEG + 1) - 1;
    constexpr int P = 14 + 3 * NK;
    // The Gaussian's SH band coefficients, read once into the thread's own column of
    // shared memory rather than from global memory in every view (blockDim = 128).
    __shared__ float s_sh[NK > 0 ? 3 * NK : 1][128];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n_pad) return;
    const int np = a.n_pad;
    const int tid = threadIdx.x;
    float G[P];
#pragma unroll
    for (int k = 0; k < P; k++) G[k] = 0.f;
    if (i < a.n) {
        float mean[3], ls[3], q[4];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            mean[k] = __ldg(a.params + (0 + k) * np + i);
            ls[k] = __ldg(a.params + (3 + k) * np + i);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) q[k] = __ldg(a.params + (6 + k) * np + i);
        // View-independent pieces: s, normalised quaternion, R(q), M = R S.
        const float s[3] = {expf(ls[0]), expf(ls[1]), expf(ls[2])};
        const float qn2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        const float qlen = fmaxf(sqrtf(qn2), 1e-12f);
        const float w = q[0] / qlen, x = q[1] / qlen, y = q[2] / qlen, z = q[3] / qlen;
        float Rq[9];
        Rq[0] = 1.f - 2.f * (y * y + z * z); Rq[1] = 2.f * (x * y - w * z); Rq[2] = 2.f * (x * z + w * y);
        Rq[3] = 2.f * (x * y + w * z); Rq[4] = 1.f - 2.f * (x * x + z * z); Rq[5] = 2.f * (y * z - w * x);
        Rq[6] = 2.f * (x * z - w * y); Rq[7] = 2.f * (y * z + w * x); Rq[8] = 1.f - 2.f * (x * x + y * y);
        float M[9], Sig[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) M[r * 3 + c] = Rq[r * 3 + c] * s[c];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++)
                Sig[r * 3 + c] = M[r * 3 + 0] * M[c * 3 + 0] + M[r * 3 + 1] * M[c * 3 + 1] + M[r * 3 + 2] * M[c * 3 + 2];
        float gSig[9];
#pragma unroll
        for (int k = 0; k < 9; k++) gSig[k] = 0.f;
        float gmean[3] = {0.f, 0.f, 0.f};
        float gnorm = 0.f;
        if (DEG > 0) {
#pragma unroll
            for (int k = 0; k < 3 * NK; k++) s_sh[k][tid] = __ldg(a.params + (14 + k) * np + i);
        }
        for (int sidx = 0; sidx < a.num_views; sidx++) {
            const size_t pair = (size_t)(a.pair_slot_first + sidx) * np + i;
            const float4 s0 = a.sg8[pair * 2 + 0];
            const float4 s1 = a.sg8[pair * 2 + 1];
            const float gC = a.sg1[pair];
            if (s0.x == 0.f && s0.y == 0.f && s0.z == 0.f && s0.w == 0.f && s1.x == 0.f && s1.y == 0.f &&
                s1.z == 0.f && s1.w == 0.f && gC == 0.f)
                continue;
            gnorm += sqrtf(s1.x * s1.x + s1.y * s1.y);  // STATS: length of (dL/du, dL/dv)
            const ViewDesc& vw = a.views[a.view_first + sidx];
            const float* W = vw.R;
            const float grgb[3] = {s0.x, s0.y, s0.z};
            G[10] += s0.w;  // opacity logit
            G[11] += grgb[0];
            G[12] += grgb[1];
            G[13] += grgb[2];
            if (DEG > 0) {
                float dvx = mean[0] - vw.campos[0], dvy = mean[1] - vw.campos[1], dvz = mean[2] - vw.campos[2];
                const float inv = rsqrtf(fmaxf(dvx * dvx + dvy * dvy + dvz * dvz, 1e-30f));
                const float dx = dvx * inv, dy = dvy * inv, dz = dvz * inv;
                float Y[NK > 0 ? NK : 1], wk[NK > 0 ? NK : 1];
                sh_basis(DEG, dx, dy, dz, Y);
#pragma unroll
                for (int k = 0; k < NK; k++) {
                    G[14 + 0 * NK + k] += Y[k] * grgb[0];
                    G[14 + 1 * NK + k] += Y[k] * grgb[1];
                    G[14 + 2 * NK + k] += Y[k] * grgb[2];
                    wk[k] = grgb[0] * s_sh[0 * NK + k][tid] + grgb[1] * s_sh[1 * NK + k][tid] +
                            grgb[2] * s_sh[2 * NK + k][tid];
                }
                float gdx, gdy, gdz;
                sh_basis_grad(DEG, dx, dy, dz, wk, gdx, gdy, gdz);
                const float dot = gdx * dx + gdy * dy + gdz * dz;
                gmean[0] += (gdx - dx * dot) * inv;
                gmean[1] += (gdy - dy * dot) * inv;
                gmean[2] += (gdz - dz * dot) * inv;
            }
            // Camera-space point.
            const float px = W[0] * mean[0] + W[1] * mean[1] + W[2] * mean[2] + vw.t[0];
            const float py = W[3] * mean[0] + W[4] * mean[1] + W[5] * mean[2] + vw.t[1];
            const float pz = W[6] * mean[0] + W[7] * mean[1] + W[8] * mean[2] + vw.t[2];
            // C = W Sigma W^T.
            float A[9], C[9];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++)
                    A[r * 3 + c] = W[r * 3 + 0] * Sig[0 * 3 + c] + W[r * 3 + 1] * Sig[1 * 3 + c] + W[r * 3 + 2] * Sig[2 * 3 + c];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++)
                    C[r * 3 + c] = A[r * 3 + 0] * W[c * 3 + 0] + A[r * 3 + 1] * W[c * 3 + 1] + A[r * 3 + 2] * W[c * 3 + 2];
            const float iz = 1.f / pz, iz2 = iz * iz;
            const float j0[3] = {vw.fx * iz, 0.f, -vw.fx * px * iz2};
            const float j1[3] = {0.f, vw.fy * iz, -vw.fy * py * iz2};
            float Cj0[3], Cj1[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                Cj0[r] = C[r * 3 + 0] * j0[0] + C[r * 3 + 2] * j0[2];
                Cj1[r] = C[r * 3 + 1] * j1[1] + C[r * 3 + 2] * j1[2];
            }
            const float ca = j0[0] * Cj0[0] + j0[2] * Cj0[2] + 0.0f;
            const float cb = j0[0] * Cj1[0] + j0[2] * Cj1[2];
            const float cc = j1[1] * Cj1[1] + j1[2] * Cj1[2];
            const float av = ca + a.dilation, bv = cb, cv = cc + a.dilation;
            const float det = av * cv - bv * bv;
            const float id2 = 1.f / (det * det);
            const float gA = s1.z, gB = s1.w, gCc = gC;
            const float gu = s1.x, gv = s1.y;
            // conic (A, B, C) = (c, -b, a) / det  ->  covariance (a, b, c).
            const float ga = (-cv * cv * gA + bv * cv * gB - bv * bv * gCc) * id2;
            const float gb = (2.f * bv * cv * gA - (det + 2.f * bv * bv) * gB + 2.f * av * bv * gCc) * id2;
            const float gc = (-bv * bv * gA + av * bv * gB - av * av * gCc) * id2;
            // a = j0' C j0, b = j0' C j1, c = j1' C j1:  dL/dC = ga j0 j0' + gb j0 j1' + gc j1 j1'.
            float GC[9];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++)
                    GC[r * 3 + c] = ga * j0[r] * j0[c] + gb * j0[r] * j1[c] + gc * j1[r] * j1[c];
            // dL/dj0 = 2 ga C j0 + gb C j1 ;  dL/dj1 = gb C j0 + 2 gc C j1.
            const float gj0_0 = 2.f * ga * Cj0[0] + gb * Cj1[0];
            const float gj0_2 = 2.f * ga * Cj0[2] + gb * Cj1[2];
            const float gj1_1 = gb * Cj0[1] + 2.f * gc * Cj1[1];
            const float gj1_2 = gb * Cj0[2] + 2.f * gc * Cj1[2];
            const float fxz2 = vw.fx * iz2, fyz2 = vw.fy * iz2;
            float gpx = gu * vw.fx * iz - gj0_2 * fxz2;
            float gpy = gv * vw.fy * iz - gj1_2 * fyz2;
            float gpz = -gu * vw.fx * px * iz2 - gv * vw.fy * py * iz2 - gj0_0 * fxz2 - gj1_1 * fyz2 +
                        gj0_2 * 2.f * vw.fx * px * iz2 * iz + gj1_2 * 2.f * vw.fy * py * iz2 * iz;
            // p = W m + t.
            gmean[0] += W[0] * gpx + W[3] * gpy + W[6] * gpz;
            gmean[1] += W[1] * gpx + W[4] * gpy + W[7] * gpz;
            gmean[2] += W[2] * gpx + W[5] * gpy + W[8] * gpz;
            // C = W Sigma W^T  ->  dL/dSigma += W^T GC W.
            float T1[9];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++)
                    T1[r * 3 + c] = GC[r * 3 + 0] * W[0 * 3 + c] + GC[r * 3 + 1] * W[1 * 3 + c] + GC[r * 3 + 2] * W[2 * 3 + c];
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++)
                    gSig[r * 3 + c] += W[0 * 3 + r] * T1[0 * 3 + c] + W[1 * 3 + r] * T1[1 * 3 + c] + W[2 * 3 + r] * T1[2 * 3 + c];
        }
        // Sigma = M M^T  ->  dL/dM = (G + G^T) M ;  M = R diag(s).
        float GM[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float acc = 0.f;
#pragma unroll
                for (int k = 0; k < 3; k++) acc += (gSig[r * 3 + k] + gSig[k * 3 + r]) * M[k * 3 + c];
                GM[r * 3 + c] = acc;
            }
        float gR[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) gR[r * 3 + c] = GM[r * 3 + c] * s[c];
#pragma unroll
        for (int c = 0; c < 3; c++)
            G[3 + c] = (GM[0 * 3 + c] * Rq[0 * 3 + c] + GM[1 * 3 + c] * Rq[1 * 3 + c] + GM[2 * 3 + c] * Rq[2 * 3 + c]) * s[c];
        // R(q^) -> q^.
        const float gw = 2.f * (-z * gR[1] + y * gR[2] + z * gR[3] - x * gR[5] - y * gR[6] + x * gR[7]);
        const float gx = 2.f * (y * gR[1] + z * gR[2] + y * gR[3] - 2.f * x * gR[4] - w * gR[5] + z * gR[6] + w * gR[7] - 2.f * x * gR[8]);
        const float gy = 2.f * (-2.f * y * gR[0] + x * gR[1] + w * gR[2] + x * gR[3] + z * gR[5] - w * gR[6] + z * gR[7] - 2.f * y * gR[8]);
        const float gz = 2.f * (-2.f * z * gR[0] - w * gR[1] + x * gR[2] + w * gR[3] - 2.f * z * gR[4] + y * gR[5] + x * gR[6] + y * gR[7]);
        // q^ = q / |q|.
        const float dq = gw * w + gx * x + gy * y + gz * z;
        G[6] = (gw - w * dq) / qlen;
        G[7] = (gx - x * dq) / qlen;
        G[8] = (gy - y * dq) / qlen;
        G[9] = (gz - z * dq) / qlen;
        G[0] = gmean[0];
        G[1] = gmean[1];
        G[2] = gmean[2];
        if (a.stats_sum && gnorm != 0.f) a.stats_sum[i] += gnorm;
    }
#pragma unroll
    for (int k = 0; k < P; k++) {
        float* dst = a.grads + (size_t)k * np + i;
        if (a.accumulate) *dst += G[k];
        else *dst = G[k];
    }
}

void launch_project_bwd(const ProjectBwdArgs& a, cudaStream_t s) {
    const int threads = 128;
    const int blocks = (a.n_pad + threads - 1) / threads;
    if (blocks == 0) return;
    switch (a.degree) {
        case 0: project_bwd_kernel<0><<<blocks, threads, 0, s>>>(a); break;
        case 1: project_bwd_kernel<1><<<blocks, threads, 0, s>>>(a); break;
        case 2: project_bwd_kernel<2><<<blocks, threads, 0, s>>>(a); break;
        default: project_bwd_kernel<3><<<blocks, threads, 0, s>>>(a); break;
    }
}

}  // namespace gs
