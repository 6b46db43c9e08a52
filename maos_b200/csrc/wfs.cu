// Geometric Shack-Hartmann WFS on the device: gradients of the atmosphere
// seen through the DMs, upstream of the reconstruction (the geometric branch
// of cuda/wfsgrad.cu gpu_wfsgrad_iwfs with gtype_sim = 0, the reference's
// default for Shack-Hartmann WFS):
//
//   OPD(p)  = sum_atm bilinear_wrap(layer, p) - sum_dm bilinear(dm, p)
//             (cuda/accphi.cu:508 gpu_atm2loc, :556 gpu_dm2loc; the point's
//             position on a map at height h: p (1 - h/hs) + h theta - v dt isim)
//   g       = GS0 OPD                       (cuda/wfsgrad.cu:458 cuspmul)
//   g      += noise                          (cuda/wfsgrad.cu:47 add_geom_noise_do)
//
// Instead of writing the OPD of every WFS point to memory and running a
// sparse product over it, one warp computes one subaperture: the OPD of the
// (nxsa+2)^2 fine-grid points its average-gradient stencil touches stays in
// registers (a band of rows at a time) and the two stencil dot
// products are reduced with warp shuffles.  A window covers only a few pixels
// of each map (OPD points are 1/64 m, layers 1/5 to 1/2 m), so the warp
// copies that block of pixels to shared memory once, interpolates each of its
// rows along x at every window column, and each point is then one
// interpolation along y between two of those rows: two shared-memory reads
// per point and map instead of four gathers.  Stencils are shared by all subapertures with the same amplitude
// neighbourhood.  The noise is two standard normals per subaperture from a
// counter-based generator (Philox4x32-10, Salmon et al. 2011) keyed by the
// seed and counted by (subaperture, WFS, step, instance), so any step of any
// instance can be drawn again.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"

namespace mb {

constexpr int kGeomMaxWfs = 16;
constexpr int kGeomMaxScr = 16;   // atmosphere layers + DMs
constexpr int kGeomWarps = 8;     // subapertures per CTA
constexpr int kGeomMaxW = 36;     // window side (nxsa + 2)
constexpr int kGeomRows = 17;    // window rows per band (OPD in registers)
constexpr int kGeomTail = (kGeomRows * (kGeomMaxW - 32) + 31) / 32;  // points of columns >= 32 per lane
constexpr int kGeomBlk = 16;     // layer pixels a window spans across, at most
constexpr int kGeomBlkStride = kGeomBlk + 1;
constexpr int kGeomHStride = kGeomMaxW;
constexpr double kGeomMaxStep = (kGeomBlk - 3.0) / (kGeomMaxW - 1.0);  // layer pixels per fine-grid step
// shared-memory bounds the kernel relies on: a band's pixel block is at most
// kGeomBlk x kGeomBlk, its interpolated rows fit the kGeomBlk x kGeomHStride
// table, and a tail point's band row fits the 8 bits it is packed in
static_assert(kGeomMaxStep * (kGeomMaxW - 1) + 3 <= kGeomBlk, "window wider than the pixel block");
static_assert(kGeomRows <= kGeomMaxW && kGeomRows < 256, "band rows");

struct GeomScr {
    const float *p;    // [ny][nx], x fastest
    long inst_stride;  // floats between instances (0: shared)
    int nx, ny;
    float alpha;
    int wrap;
};
struct GeomWfsT {
    int nsa, nxsa, sa_off;
    long g_off;
};
struct GeomCoef {  // screen index = fine-grid index * s + b (before the wind shift)
    double sx, bx, sy, by;
};
struct GeomTab {
    int nwfs, nscr, natm;
    GeomWfsT w[kGeomMaxWfs];
    GeomScr s[kGeomMaxScr];
    GeomCoef c[kGeomMaxWfs][kGeomMaxScr];
};

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const unsigned lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// grid: (ceil(max nsa / kGeomWarps), nwfs, nbatch); block: kGeomWarps warps.
// sa_ix/sa_iy: fine-grid index of each subaperture's first point; sa_st its
// stencil; st_off the offset of each stencil ([2][W*W] floats) in st; nea
// per WFS [3][nsa] (sqrt-NEA xx, yy, xy) at 3*sa_off; wind_px: per instance and
// atmosphere layer, the shift in layer pixels per step (v dt / dx).
__global__ void __launch_bounds__(kGeomWarps * 32, 4)
k_wfs_geom(const __grid_constant__ GeomTab t, const int *__restrict__ sa_ix, const int *__restrict__ sa_iy,
           const int *__restrict__ sa_st, const float *__restrict__ st, const long *__restrict__ st_off,
           const float *__restrict__ nea, const double2 *__restrict__ wind_px, float *__restrict__ grad,
           long grad_stride, long isim, unsigned long long seed) {
    __shared__ int4 sbase[kGeomWarps][kGeomMaxScr];
    __shared__ float sblk[kGeomWarps][kGeomBlk * kGeomBlkStride];
    __shared__ float shx[kGeomWarps][kGeomBlk * kGeomHStride];
    __shared__ float2 srow[kGeomWarps][kGeomRows];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int iw = blockIdx.y, inst = blockIdx.z;
    const GeomWfsT &W = t.w[iw];
    const int isa = blockIdx.x * kGeomWarps + wid;
    if (isa >= W.nsa) return;  // the whole warp: no block-wide barrier below
    const int gi = W.sa_off + isa;
    const int wn = W.nxsa + 2, npts = wn * wn;
    const int gx0 = sa_ix[gi] - 1, gy0 = sa_iy[gi] - 1;
    // each map's position of the window's first point: integer part (wrapped
    // for the atmosphere) and fraction
    if (lane < t.nscr) {
        const GeomCoef c = t.c[iw][lane];
        const GeomScr &S = t.s[lane];
        double u = fma((double)gx0, c.sx, c.bx), v = fma((double)gy0, c.sy, c.by);
        if (lane < t.natm) {  // frozen flow: the layer moves by v dt per step
            const double2 w = wind_px[(long)inst * t.natm + lane];
            u = fma(-w.x, (double)isim, u);
            v = fma(-w.y, (double)isim, v);
        }
        const double fu = floor(u), fv = floor(v);
        long long iu = (long long)fmin(fmax(fu, -1e9), 1e9), iv = (long long)fmin(fmax(fv, -1e9), 1e9);
        if (S.wrap) {
            iu %= S.nx;
            if (iu < 0) iu += S.nx;
            iv %= S.ny;
            if (iv < 0) iv += S.ny;
        }
        sbase[wid][lane] = make_int4((int)iu, (int)iv, __float_as_int((float)(u - fu)), __float_as_int((float)(v - fv)));
    }
    __syncwarp();
    const float *__restrict__ w = st + st_off[sa_st[gi]];
    float *blk = sblk[wid], *hx = shx[wid];
    float gx = 0.f, gy = 0.f;
    // Lane c owns window column c (< 32) of a band of kGeomRows rows; the
    // points of the columns from 32 on (wn > 32: at most 4 columns) are dealt
    // out over the lanes, kGeomTail at most each.  OPD of the band stays in
    // registers.
    const int ntail = wn > 32 ? wn - 32 : 0;
    const bool main_ok = lane < wn;
    for (int r0 = 0; r0 < wn; r0 += kGeomRows) {
        const int nr = min(kGeomRows, wn - r0);
        float opd[kGeomRows];
#pragma unroll
        for (int j = 0; j < kGeomRows; j++) opd[j] = 0.f;
        float opdt[kGeomTail];
        int tpk[kGeomTail];  // band row << 8 | column of each tail point, -1: none
#pragma unroll
        for (int q = 0; q < kGeomTail; q++) {
            const int tp = lane + 32 * q;
            opdt[q] = 0.f;
            tpk[q] = tp < nr * ntail ? (tp / ntail) << 8 | (32 + tp % ntail) : -1;
        }
        for (int s = 0; s < t.nscr; s++) {
            const GeomScr S = t.s[s];
            const int4 b = sbase[wid][s];
            const float sxf = (float)t.c[iw][s].sx, syf = (float)t.c[iw][s].sy;
            const float fu0 = __int_as_float(b.z), fv0 = __int_as_float(b.w);
            const float *__restrict__ P = S.p + (long)inst * S.inst_stride;
            // the layer pixels this band touches: columns 0..nbu-1 and rows
            // v0..v0+nbv-1 from the window origin's pixel (the +1 neighbours included)
            const int v0 = (int)floorf(fmaf((float)r0, syf, fv0));
            const int nbv = min((int)floorf(fmaf((float)(r0 + nr - 1), syf, fv0)) + 2 - v0, kGeomBlk);
            const int nbu = min((int)floorf(fmaf((float)(wn - 1), sxf, fu0)) + 2, kGeomBlk);
            const float inv_nbu = __frcp_rn((float)nbu);
            __syncwarp();  // the previous map's tables are no longer read
            for (int e = lane; e < nbu * nbv; e += 32) {
                const int bv = (int)(((float)e + 0.5f) * inv_nbu), bu = e - bv * nbu;
                int c = b.x + bu, r = b.y + v0 + bv;
                float val = 0.f;
                if (S.wrap) {
                    c -= c >= S.nx ? S.nx : 0;
                    r -= r >= S.ny ? S.ny : 0;
                    val = __ldg(P + (long)r * S.nx + c);
                } else {
                    c = c == S.nx ? 0 : c;  // the +1 neighbour of the last column is column 0
                    r = r == S.ny ? 0 : r;
                    if (c >= 0 && c < S.nx && r >= 0 && r < S.ny) val = __ldg(P + (long)r * S.nx + c);
                }
                blk[bv * kGeomBlkStride + bu] = val;
            }
            __syncwarp();
            // each block row interpolated along x at every window column
            for (int cc = lane; cc < wn; cc += 32) {
                const float uf = fmaf((float)cc, sxf, fu0), fl = floorf(uf), ax = uf - fl;
                const int lu = (int)fl;
                const bool ok = S.wrap || (b.x + lu >= 0 && b.x + lu < S.nx);  // off the map: no contribution
                for (int bv = 0; bv < nbv; bv++) {
                    const float m0 = blk[bv * kGeomBlkStride + lu], m1 = blk[bv * kGeomBlkStride + lu + 1];
                    hx[bv * kGeomHStride + cc] = ok ? fmaf(m1 - m0, ax, m0) : 0.f;
                }
            }
            // each band row's pair of interpolated rows (offset in hx, -1 when
            // the row is off the map) and its fraction along y
            for (int rr = lane; rr < nr; rr += 32) {  // every band row, whatever kGeomRows is
                const float vf = fmaf((float)(r0 + rr), syf, fv0), flv = floorf(vf);
                const int lv = (int)flv - v0;
                const bool rok = S.wrap || (b.y + (int)flv >= 0 && b.y + (int)flv < S.ny);
                srow[wid][rr] = make_float2(__int_as_float(rok && lv >= 0 && lv + 1 < nbv ? lv * kGeomHStride : -1),
                                            vf - flv);
            }
            __syncwarp();
            // every point of the band: along y between two of those rows
#pragma unroll
            for (int j = 0; j < kGeomRows; j++) {
                if (j < nr && main_ok) {
                    const float2 q = srow[wid][j];
                    const int off = __float_as_int(q.x);
                    if (off >= 0) {
                        const float h0 = hx[off + lane], h1 = hx[off + kGeomHStride + lane];
                        opd[j] = fmaf(S.alpha, fmaf(h1 - h0, q.y, h0), opd[j]);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < kGeomTail; q++) {
                if (tpk[q] >= 0) {
                    const int tc = tpk[q] & 255;
                    const float2 rq = srow[wid][tpk[q] >> 8];
                    const int off = __float_as_int(rq.x);
                    if (off >= 0) {
                        const float h0 = hx[off + tc], h1 = hx[off + kGeomHStride + tc];
                        opdt[q] = fmaf(S.alpha, fmaf(h1 - h0, rq.y, h0), opdt[q]);
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kGeomRows; j++) {
            if (j < nr && main_ok) {
                const int k = (r0 + j) * wn + lane;
                gx = fmaf(__ldg(w + k), opd[j], gx);
                gy = fmaf(__ldg(w + npts + k), opd[j], gy);
            }
        }
#pragma unroll
        for (int q = 0; q < kGeomTail; q++) {
            if (tpk[q] >= 0) {
                const int k = (r0 + (tpk[q] >> 8)) * wn + (tpk[q] & 255);
                gx = fmaf(__ldg(w + k), opdt[q], gx);
                gy = fmaf(__ldg(w + npts + k), opdt[q], gy);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
        gy += __shfl_xor_sync(0xffffffffu, gy, o);
    }
    if (lane == 0) {
        if (seed) {
            const uint4 o = philox4x32_10(make_uint4((unsigned)isa, (unsigned)iw, (unsigned)isim, (unsigned)inst),
                                          make_uint2((unsigned)seed, (unsigned)(seed >> 32)));
            const double u1 = ((double)o.x + 1.0) * 0x1p-32, u2 = (double)o.y * 0x1p-32;
            const double rr = sqrt(-2.0 * log(u1));
            double sn, cs;
            sincospi(2.0 * u2, &sn, &cs);
            const float n1 = (float)(rr * cs), n2 = (float)(rr * sn);
            const float *ne = nea + 3L * W.sa_off;
            gx = fmaf(n1, ne[isa], gx);
            gy = fmaf(n2, ne[W.nsa + isa], fmaf(n1, ne[2 * W.nsa + isa], gy));
        }
        float *g = grad + (long)inst * grad_stride + W.g_off;
        g[isa] = gx;
        g[W.nsa + isa] = gy;
    }
}

struct GeomWfsHost {
    int nwfs = 0, natm = 0, ndm = 0, nbatch = 1;
    long ngrad = 0, nact = 0, atm_stride = 0;
    int max_nsa = 0;
    double dt = 0;
    std::vector<int> nsa, nxsa;
    std::vector<double> dx, gox, goy, thetax, thetay, hs;
    std::vector<int> anx, any;
    std::vector<double> adx, aox, aoy, aht;
    std::vector<double> wind;  // [nbatch][natm][2] m/s
    std::vector<long> aoff;  // layer offsets within one instance
    std::vector<int> dnx, dny;
    std::vector<double> ddx, dox, doy, dht;
    std::vector<long> doff;  // DM offsets within one instance's commands
    DevBuf<int> sa_ix, sa_iy, sa_st;
    DevBuf<float> st, nea, atm;
    DevBuf<double2> wind_px;
    void upload_wind() {
        std::vector<double2> w((size_t)nbatch * natm);
        for (int i = 0; i < nbatch; i++)
            for (int l = 0; l < natm; l++) {
                const size_t k = (size_t)i * natm + l;
                w[k] = make_double2(wind[2 * k] * dt / adx[l], wind[2 * k + 1] * dt / adx[l]);
            }
        wind_px.upload(w);
    }
    DevBuf<long> st_off;
    bool have_nea = false;
};

}  // namespace mb

struct mb_geom_wfs {
    mb::GeomWfsHost H;
};

extern "C" {

int mb_geom_wfs_create(const mb_geom_wfs_desc *d, mb_geom_wfs **out) {
    using namespace mb;
    if (!out || !d || d->nwfs < 1 || d->nwfs > kGeomMaxWfs || d->natm < 0 || d->ndm < 0 ||
        d->natm + d->ndm > kGeomMaxScr || d->nbatch < 1 || !d->nsa || !d->nxsa || !d->dx || !d->gox || !d->goy ||
        !d->thetax || !d->thetay || !d->hs || !d->sa_ix || !d->sa_iy || !d->sa_stencil || d->nstencil < 1 ||
        !d->stencil_off || !d->stencils || d->stencil_len < 1 ||
        (d->natm && (!d->atm_nx || !d->atm_ny || !d->atm_dx || !d->atm_ox || !d->atm_oy || !d->atm_ht ||
                     !d->atm_vx || !d->atm_vy)) ||
        (d->ndm && (!d->dm_nx || !d->dm_ny || !d->dm_dx || !d->dm_ox || !d->dm_oy || !d->dm_ht))) {
        set_error("mb_geom_wfs_create: invalid descriptor");
        return MB_EINVAL;
    }
    *out = nullptr;
    mb_geom_wfs *h = new (std::nothrow) mb_geom_wfs();
    if (!h) return MB_ENOMEM;
    try {
        GeomWfsHost &H = h->H;
        H.nwfs = d->nwfs;
        H.natm = d->natm;
        H.ndm = d->ndm;
        H.nbatch = d->nbatch;
        H.dt = d->dt;
        long nsa_tot = 0;
        for (int i = 0; i < d->nwfs; i++) {
            if (d->nsa[i] < 1 || d->nxsa[i] < 1 || d->nxsa[i] + 2 > kGeomMaxW || !(d->dx[i] > 0)) {
                set_error("mb_geom_wfs_create: WFS %d: nsa %d, nxsa %d (window at most %d points across)", i,
                          d->nsa[i], d->nxsa[i], kGeomMaxW);
                throw InvalidArg{MB_EINVAL};
            }
            H.nsa.push_back(d->nsa[i]);
            H.nxsa.push_back(d->nxsa[i]);
            H.dx.push_back(d->dx[i]);
            H.gox.push_back(d->gox[i]);
            H.goy.push_back(d->goy[i]);
            H.thetax.push_back(d->thetax[i]);
            H.thetay.push_back(d->thetay[i]);
            H.hs.push_back(d->hs[i]);
            nsa_tot += d->nsa[i];
            H.ngrad += 2L * d->nsa[i];
            if (d->nsa[i] > H.max_nsa) H.max_nsa = d->nsa[i];
        }
        std::vector<int> ix(d->sa_ix, d->sa_ix + nsa_tot), iy(d->sa_iy, d->sa_iy + nsa_tot),
            sid(d->sa_stencil, d->sa_stencil + nsa_tot);
        std::vector<long> soff(d->stencil_off, d->stencil_off + d->nstencil);
        // every subaperture's stencil must be one of its WFS's size and inside the table
        long k = 0;
        for (int i = 0; i < d->nwfs; i++) {
            const long len = 2L * (d->nxsa[i] + 2) * (d->nxsa[i] + 2);
            for (int j = 0; j < d->nsa[i]; j++, k++) {
                if (sid[k] < 0 || sid[k] >= d->nstencil || soff[sid[k]] < 0 || soff[sid[k]] + len > d->stencil_len ||
                    ix[k] < 1 || iy[k] < 1) {
                    set_error("mb_geom_wfs_create: subaperture %d of WFS %d: stencil %d or grid index out of range",
                              j, i, sid[k]);
                    throw InvalidArg{MB_EINVAL};
                }
            }
        }
        H.sa_ix.upload(ix);
        H.sa_iy.upload(iy);
        H.sa_st.upload(sid);
        H.st_off.upload(soff);
        std::vector<float> stf(d->stencils, d->stencils + d->stencil_len);
        H.st.upload(stf);
        if (d->nea) {
            std::vector<float> nf(d->nea, d->nea + 3 * nsa_tot);
            H.nea.upload(nf);
            H.have_nea = true;
        }
        for (int l = 0; l < d->natm; l++) {
            if (d->atm_nx[l] < 2 || d->atm_ny[l] < 2 || !(d->atm_dx[l] > 0)) {
                set_error("mb_geom_wfs_create: atmosphere layer %d: %d x %d", l, d->atm_nx[l], d->atm_ny[l]);
                throw InvalidArg{MB_EINVAL};
            }
            // a window must span at most kGeomBlk layer pixels (and fewer than the layer has)
            for (int i = 0; i < d->nwfs; i++) {
                const double sc = std::isfinite(d->hs[i]) ? 1.0 - d->atm_ht[l] / d->hs[i] : 1.0;
                const double step = d->dx[i] * sc / d->atm_dx[l];
                if (!(sc > 0) || step > kGeomMaxStep || kGeomBlk >= d->atm_nx[l] || kGeomBlk >= d->atm_ny[l]) {
                    set_error("mb_geom_wfs_create: layer %d: WFS %d steps %.3g layer pixels per OPD point "
                              "(at most %.3g) on a %d x %d layer", l, i, step, kGeomMaxStep, d->atm_nx[l],
                              d->atm_ny[l]);
                    throw InvalidArg{MB_EUNSUP};
                }
            }
            H.anx.push_back(d->atm_nx[l]);
            H.any.push_back(d->atm_ny[l]);
            H.adx.push_back(d->atm_dx[l]);
            H.aox.push_back(d->atm_ox[l]);
            H.aoy.push_back(d->atm_oy[l]);
            H.aht.push_back(d->atm_ht[l]);
            H.aoff.push_back(H.atm_stride);
            H.atm_stride += (long)d->atm_nx[l] * d->atm_ny[l];
        }
        for (int m = 0; m < d->ndm; m++) {
            if (d->dm_nx[m] < 2 || d->dm_ny[m] < 2 || !(d->dm_dx[m] > 0)) {
                set_error("mb_geom_wfs_create: DM %d: %d x %d", m, d->dm_nx[m], d->dm_ny[m]);
                throw InvalidArg{MB_EINVAL};
            }
            for (int i = 0; i < d->nwfs; i++) {
                const double sc = std::isfinite(d->hs[i]) ? 1.0 - d->dm_ht[m] / d->hs[i] : 1.0;
                const double step = d->dx[i] * sc / d->dm_dx[m];
                if (!(sc > 0) || step > kGeomMaxStep) {
                    set_error("mb_geom_wfs_create: DM %d: WFS %d steps %.3g actuators per OPD point (at most %.3g)",
                              m, i, step, kGeomMaxStep);
                    throw InvalidArg{MB_EUNSUP};
                }
            }
            H.dnx.push_back(d->dm_nx[m]);
            H.dny.push_back(d->dm_ny[m]);
            H.ddx.push_back(d->dm_dx[m]);
            H.dox.push_back(d->dm_ox[m]);
            H.doy.push_back(d->dm_oy[m]);
            H.dht.push_back(d->dm_ht[m]);
            H.doff.push_back(H.nact);
            H.nact += (long)d->dm_nx[m] * d->dm_ny[m];
        }
        H.wind.resize((size_t)H.nbatch * H.natm * 2);
        for (int i = 0; i < H.nbatch; i++)
            for (int l = 0; l < H.natm; l++) {
                H.wind[2 * ((size_t)i * H.natm + l)] = d->atm_vx[l];
                H.wind[2 * ((size_t)i * H.natm + l) + 1] = d->atm_vy[l];
            }
        if (H.natm) H.upload_wind();
        if (H.atm_stride) {
            H.atm.alloc((size_t)H.atm_stride * H.nbatch);
            H.atm.zero_async(nullptr);
        }
        MB_CUDA_TRY(cudaDeviceSynchronize());
    } catch (const CudaError &e) {
        delete h;
        return e.code;
    } catch (const InvalidArg &e) {
        delete h;
        return e.code;
    }
    *out = h;
    return MB_OK;
}

void mb_geom_wfs_free(mb_geom_wfs *h) { delete h; }

long mb_geom_wfs_ngrad(const mb_geom_wfs *h) { return h ? h->H.ngrad : -1; }
long mb_geom_wfs_nact(const mb_geom_wfs *h) { return h ? h->H.nact : -1; }

int mb_geom_wfs_set_atm(mb_geom_wfs *h, int inst, int layer, const double *screen) {
    if (!h || !screen || inst < 0 || inst >= h->H.nbatch || layer < 0 || layer >= h->H.natm) {
        mb::set_error("mb_geom_wfs_set_atm: invalid arguments");
        return MB_EINVAL;
    }
    try {
        mb::GeomWfsHost &H = h->H;
        const long n = (long)H.anx[layer] * H.any[layer];
        std::vector<float> f(screen, screen + n);
        MB_CUDA_TRY(cudaMemcpy(H.atm.p + (size_t)inst * H.atm_stride + H.aoff[layer], f.data(), n * sizeof(float),
                               cudaMemcpyHostToDevice));
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

int mb_geom_wfs_set_wind(mb_geom_wfs *h, int inst, int layer, double vx, double vy) {
    if (!h || inst < 0 || inst >= h->H.nbatch || layer < 0 || layer >= h->H.natm) {
        mb::set_error("mb_geom_wfs_set_wind: invalid arguments");
        return MB_EINVAL;
    }
    try {
        mb::GeomWfsHost &H = h->H;
        H.wind[2 * ((size_t)inst * H.natm + layer)] = vx;
        H.wind[2 * ((size_t)inst * H.natm + layer) + 1] = vy;
        H.upload_wind();
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

int mb_geom_wfs_grad(mb_geom_wfs *h, long isim, const float *d_dm, float *d_grad, unsigned long long seed,
                     void *stream) {
    using namespace mb;
    if (!h || !d_grad || isim < 0 || (seed && !h->H.have_nea)) {
        set_error("mb_geom_wfs_grad: invalid arguments%s", h && seed && !h->H.have_nea ? " (no NEA tables)" : "");
        return MB_EINVAL;
    }
    try {
        const GeomWfsHost &H = h->H;
        GeomTab t;
        std::memset(&t, 0, sizeof(t));
        t.nwfs = H.nwfs;
        int ns = 0;
        for (int l = 0; l < H.natm; l++, ns++)
            t.s[ns] = GeomScr{H.atm.p + H.aoff[l], H.atm_stride, H.anx[l], H.any[l], 1.0f, 1};
        if (d_dm)
            for (int m = 0; m < H.ndm; m++, ns++)
                t.s[ns] = GeomScr{d_dm + H.doff[m], H.nact, H.dnx[m], H.dny[m], -1.0f, 0};
        t.nscr = ns;
        t.natm = H.natm;
        long goff = 0;
        int saoff = 0;
        for (int i = 0; i < H.nwfs; i++) {
            t.w[i] = GeomWfsT{H.nsa[i], H.nxsa[i], saoff, goff};
            saoff += H.nsa[i];
            goff += 2L * H.nsa[i];
            for (int s = 0; s < ns; s++) {
                const bool atm = s < H.natm;
                const int q = atm ? s : s - H.natm;
                const double ht = atm ? H.aht[q] : H.dht[q];
                const double sdx = atm ? H.adx[q] : H.ddx[q];
                const double sox = atm ? H.aox[q] : H.dox[q], soy = atm ? H.aoy[q] : H.doy[q];
                const double sc = std::isfinite(H.hs[i]) ? 1.0 - ht / H.hs[i] : 1.0;
                const double dispx = ht * H.thetax[i], dispy = ht * H.thetay[i];
                t.c[i][s] = GeomCoef{H.dx[i] * sc / sdx, (H.gox[i] * sc + dispx - sox) / sdx, H.dx[i] * sc / sdx,
                                     (H.goy[i] * sc + dispy - soy) / sdx};
            }
        }
        const dim3 grid((unsigned)((H.max_nsa + kGeomWarps - 1) / kGeomWarps), (unsigned)H.nwfs, (unsigned)H.nbatch);
        k_wfs_geom<<<grid, kGeomWarps * 32, 0, (cudaStream_t)stream>>>(t, H.sa_ix.p, H.sa_iy.p, H.sa_st.p, H.st.p,
                                                                      H.st_off.p, H.nea.p, H.wind_px.p, d_grad,
                                                                      H.ngrad, isim, seed);
        MB_CHECK_LAUNCH();
    } catch (const CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

}  // extern "C"
