// Tensor-core 3x3 convolutions (tc_conv.cuh) on the host side: tensor maps,
// launch shapes, and C-ABI entry points that run one convolution on host buffers (the
// parity tests drive the kernels through them).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "cfm_internal.h"
#include "tc_conv.cuh"
#include "unet_fused.cuh"
#include "unet_internal.h"

namespace cfm {

namespace {

int encode_map(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims,
               const cuuint64_t *strides, const cuuint32_t *box, int sw_bytes) {
    auto enc = tensor_map_encoder();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled is unavailable");
        return CFM_UNSUPPORTED;
    }
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, rank, const_cast<void *>(base), dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           sw_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return CFM_BAD_ARG;
    }
    return CFM_OK;
}

constexpr int round1k(int v) { return (v + 1023) / 1024 * 1024; }
// Dynamic shared memory of one CTA alone on an SM (the 227 KB a block may
// opt into, less its static part and some slack); two CTAs take half each.
constexpr int TC_SMEM_MAX = 220 * 1024;

// Shared-memory plan of one pass: ring depth and slot size, resident
// weights, CTAs per SM.  Two CTAs share an SM when the grid has at least two
// tiles per SM and both fit (shared memory, 512 TMEM columns); the weights
// stay resident when a CTA runs at least two tiles and they leave room for
// three slots.
template <int KC, int N>
int plan_kc_n(TcConvParams &p, int num_sms, int *cps_out) {
    constexpr int SW = KC * 2, BTAP = N * SW;
    const bool conv = p.mode == 0;
    if (conv) {
        // split-K when the pixel tiles leave SMs idle: at least one halo step
        // (three taps) or two per-tap steps per split, within the workspace
        const int ptiles = p.tiles_x * p.tiles_y * p.B;
        const long long npix = (long long)p.B * p.H * p.W;
        int S = ptiles < num_sms ? num_sms / ptiles : 1;
        S = std::min(S, p.ksteps / (p.halo ? 1 : 2));
        if (p.ws_floats > 0) S = (int)std::min<long long>(S, p.ws_floats / (npix * N));
        else S = 1;
        p.csplit = std::max(S, 1);
        p.ntiles = ptiles * p.csplit;
    }
    p.a_region = conv && p.halo ? round1k(136 * SW) : 128 * SW;
    const int b_stage = conv && p.halo ? 3 * BTAP : BTAP;
    const int wbytes = conv ? round1k(9 * p.nch * BTAP) : 0;
    // (a weight gradient's split is planned for up to two tiles per SM)
    const int cps =
        (2 * tc_tmem_cols<N>() <= 512 && p.ntiles >= (conv ? 2 * num_sms : num_sms + 1)) ? 2 : 1;
    // per-CTA dynamic shared memory (the SM has 228 KB; 1 KB per CTA is reserved)
    const int budget = cps == 2 ? TC_SMEM_MAX / 2 : TC_SMEM_MAX;
    const int overhead = 1024 + 8 * 8 + 16;
    const long long tiles_per_cta = (p.ntiles + (long long)num_sms * cps - 1) / ((long long)num_sms * cps);
    p.wres = conv && tiles_per_cta >= 2 && wbytes + 3 * (p.a_region + 16) + overhead <= budget;
    p.wres_bytes = p.wres ? wbytes : 0;
    p.stage_bytes = p.wres ? p.a_region : round1k(p.a_region + b_stage);
    int stages = (budget - overhead - p.wres_bytes) / (p.stage_bytes + 16);
    if (stages < 2 && conv && p.halo) {
        // wide streamed weights: three taps per slot do not fit twice, go per tap
        p.halo = 0;
        p.ksteps = 9 * p.nch;
        return plan_kc_n<KC, N>(p, num_sms, cps_out);  // (re-plans the split too)
    }
    stages = std::min(stages, 16);
    if (stages < 2) {
        set_error("tensor-core convolution: no shared-memory plan for KC %d, N %d", KC, N);
        return CFM_UNSUPPORTED;
    }
    p.stages = stages;
    *cps_out = cps;
    return CFM_OK;
}

template <int KC, int N>
int launch_kc_n(const CUtensorMap &a0, const CUtensorMap &a1, const CUtensorMap &b, TcConvParams p,
                cudaStream_t s) {
    static std::once_flag once[64];
    static cudaError_t attr_err[64];
    int dev = 0;
    CFM_CUDA_TRY(cudaGetDevice(&dev));
    std::call_once(once[dev & 63], [&] {
        attr_err[dev & 63] = cudaFuncSetAttribute(tc_conv_kernel<KC, N>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_MAX);
        if (attr_err[dev & 63] == cudaSuccess)
            attr_err[dev & 63] = cudaFuncSetAttribute(
                tc_conv_kernel<KC, N>, cudaFuncAttributePreferredSharedMemoryCarveout,
                (int)cudaSharedmemCarveoutMaxShared);
    });
    CFM_CUDA_TRY(attr_err[dev & 63]);
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    int cps = 1;
    if ((st = plan_kc_n<KC, N>(p, di.num_sms, &cps))) return st;
    const size_t smem = tc_conv_smem(p.wres_bytes, p.stages, p.stage_bytes);
    // (the occupancy query under-reports two CTAs of ~110 KB; the plan keeps
    // 2 x (dynamic + static + 1 KB reserved) inside the SM's 228 KB)
    const int grid = std::min(p.ntiles, di.num_sms * cps);
    CFM_CUDA_TRY(launch_pdl(tc_conv_kernel<KC, N>, dim3(grid), dim3(192), smem, s, a0, a1, b, p));
    if (p.mode == 0 && p.csplit > 1) {
        const long long npix = (long long)p.B * p.H * p.W;
        const long long items = npix * (N / 8);
        const int blocks = (int)std::min<long long>((items + 255) / 256, (long long)di.num_sms * 8);
        CFM_CUDA_TRY(launch_pdl(tc_splitk_epilogue<N>, dim3(blocks), dim3(256), 0, s, (const float *)p.ws,
                                p.csplit, npix, p.bias, p.relu, p.mask, p.out));
    }
    return CFM_OK;
}

template <int KC>
int launch_kc(int n, const CUtensorMap &a0, const CUtensorMap &a1, const CUtensorMap &b,
              const TcConvParams &p, cudaStream_t s) {
    switch (n) {
        case 32: return launch_kc_n<KC, 32>(a0, a1, b, p, s);
        case 64: return launch_kc_n<KC, 64>(a0, a1, b, p, s);
        case 128: return launch_kc_n<KC, 128>(a0, a1, b, p, s);
        case 256: return launch_kc_n<KC, 256>(a0, a1, b, p, s);
        default: set_error("unsupported channel count %d", n); return CFM_UNSUPPORTED;
    }
}

int launch(int kc, int n, const CUtensorMap &a0, const CUtensorMap &a1, const CUtensorMap &b,
           const TcConvParams &p, cudaStream_t s) {
    return kc == 64 ? launch_kc<64>(n, a0, a1, b, p, s) : launch_kc<32>(n, a0, a1, b, p, s);
}

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

}  // namespace

namespace {

// The parameters of a convolution pass before its launch plan: tiling (a
// 128-pixel tile is bx x by), channel chunk, halo or per-tap staging, the
// epilogue and the split-K workspace.
int conv_fwd_params(const ConvArgs &a, TcConvParams &p, int *kc_out) {
    CFM_ARG_CHECK(a.Cin % 32 == 0 && a.Cin <= 256, "Cin must be a multiple of 32, at most 256");
    CFM_ARG_CHECK(a.Cout == 32 || a.Cout == 64 || a.Cout == 128 || a.Cout == 256, "Cout");
    CFM_ARG_CHECK(a.W % 128 == 0 || (pow2(a.W) && a.W <= 128), "W: a power of two or a multiple of 128");
    CFM_ARG_CHECK(a.H >= 1 && a.B >= 1, "H, B");
    const int kc = a.Cin % 64 == 0 ? 64 : 32;
    p = TcConvParams{};
    p.mode = 0;
    p.B = a.B;
    p.H = a.H;
    p.W = a.W;
    p.Cin = a.Cin;
    p.Cout = a.Cout;
    p.bx = std::min(a.W, 128);
    p.by = 128 / p.bx;
    p.tiles_x = (a.W + p.bx - 1) / p.bx;
    p.tiles_y = (a.H + p.by - 1) / p.by;
    p.ntiles = p.tiles_x * p.tiles_y * a.B;
    p.nch = a.Cin / kc;
    p.halo = p.bx == 128;
    p.ksteps = (p.halo ? 3 : 9) * p.nch;
    p.bias = a.bias;
    p.relu = a.relu;
    p.mask = a.mask;
    p.out = a.out;
    p.err = a.err;
    p.ws = a.ws;
    p.ws_floats = a.ws ? a.ws_floats : 0;
    p.csplit = 1;
    p.budget_ns = barrier_timeout_ns();
    *kc_out = kc;
    return CFM_OK;
}

// Its tensor maps: per-tap boxes (bx x by pixels), halo boxes (130 pixels of
// one row; the per-tap map when the tile is narrower) and the weights.
int conv_fwd_maps(const ConvArgs &a, const TcConvParams &p, int kc, CUtensorMap *ma, CUtensorMap *mh,
                  CUtensorMap *mb) {
    const cuuint64_t da[4] = {(cuuint64_t)a.Cin, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
    const cuuint64_t sa[3] = {(cuuint64_t)a.Cin * 2, (cuuint64_t)a.W * a.Cin * 2,
                              (cuuint64_t)a.H * a.W * a.Cin * 2};
    const cuuint32_t ba[4] = {(cuuint32_t)kc, (cuuint32_t)p.bx, (cuuint32_t)p.by, 1};
    int st = encode_map(ma, a.x, 4, da, sa, ba, kc * 2);
    if (st) return st;
    *mh = *ma;
    if (p.halo) {
        const cuuint32_t bh[4] = {(cuuint32_t)kc, (cuuint32_t)TC_HALO_ROWS, 1, 1};
        if ((st = encode_map(mh, a.x, 4, da, sa, bh, kc * 2))) return st;
    }
    const cuuint64_t db[3] = {(cuuint64_t)a.Cin, (cuuint64_t)a.Cout, 9};
    const cuuint64_t sb[2] = {(cuuint64_t)a.Cin * 2, (cuuint64_t)a.Cout * a.Cin * 2};
    const cuuint32_t bb[3] = {(cuuint32_t)kc, (cuuint32_t)a.Cout, 1};
    return encode_map(mb, a.w, 3, db, sb, bb, kc * 2);
}

template <int KC>
int plan_kc(int n, TcConvParams &p, int num_sms, int *cps) {
    switch (n) {
        case 32: return plan_kc_n<KC, 32>(p, num_sms, cps);
        case 64: return plan_kc_n<KC, 64>(p, num_sms, cps);
        case 128: return plan_kc_n<KC, 128>(p, num_sms, cps);
        case 256: return plan_kc_n<KC, 256>(p, num_sms, cps);
        default: set_error("unsupported channel count %d", n); return CFM_UNSUPPORTED;
    }
}

}  // namespace

int tc_conv_fwd(const ConvArgs &a, cudaStream_t s) {
    TcConvParams p;
    int kc = 0;
    int st = conv_fwd_params(a, p, &kc);
    if (st) return st;
    CUtensorMap ma, mh, mb;
    if ((st = conv_fwd_maps(a, p, kc, &ma, &mh, &mb))) return st;
    return launch(kc, a.Cout, ma, mh, mb, p, s);
}

int unet_forward_fused(const FusedForwardArgs &f, cudaStream_t s) {
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    UfParams p{};
    UfMaps m;
    int slot = 0;
    for (int l = 0; l < UF_CONVS; ++l) {
        const ConvArgs &a = f.conv[l];
        TcConvParams tp;
        int kc = 0, cps = 1;
        if ((st = conv_fwd_params(a, tp, &kc))) return st;
        CUtensorMap ma, mh, mb;
        if ((st = conv_fwd_maps(a, tp, kc, &ma, &mh, &mb))) return st;
        // the per-layer launch plan: the same staging and split-K, so the
        // same K order and partial sums
        if ((st = kc == 64 ? plan_kc<64>(a.Cout, tp, di.num_sms, &cps) : plan_kc<32>(a.Cout, tp, di.num_sms, &cps)))
            return st;
        UfConv &L = p.conv[l];
        L.H = a.H;
        L.W = a.W;
        L.N = a.Cout;
        L.kc = kc;
        L.bx = tp.bx;
        L.by = tp.by;
        L.tiles_x = tp.tiles_x;
        L.tiles_y = tp.tiles_y;
        L.nch = tp.nch;
        L.halo = tp.halo;
        L.ksteps = tp.ksteps;
        L.csplit = tp.csplit;
        L.ntiles = tp.ntiles;
        L.a_region = tp.a_region;
        L.bias = a.bias;
        L.relu = a.relu;
        L.out = a.out;
        L.ws = a.ws;
        L.skip = f.skip[l];
        L.uout = f.uout[l];
        m.a[l] = tp.halo ? mh : ma;
        m.b[l] = mb;
        const int b_stage = (tp.halo ? 3 : 1) * a.Cout * kc * 2;
        slot = std::max(slot, round1k(tp.a_region + b_stage));
    }
    int stages = 2;
    while (stages < 16 && uf_smem_bytes(stages + 1, slot) <= (size_t)TC_SMEM_MAX) ++stages;
    if (uf_smem_bytes(stages, slot) > (size_t)TC_SMEM_MAX) {
        set_error("persistent U-Net forward: a %d-byte ring slot leaves no two-stage ring", slot);
        return CFM_UNSUPPORTED;
    }
    p.B = f.B;
    p.H = f.H;
    p.W = f.W;
    p.x = f.x;
    p.out = f.out;
    p.in_scale = f.in_scale;
    p.cin_w = f.cin_w;
    p.cin_b = f.cin_b;
    p.cout_w = f.cout_w;
    p.cout_b = f.cout_b;
    p.h0 = f.h0;
    p.p1 = f.p1;
    p.h1 = f.h1;
    p.p2 = f.p2;
    p.h2 = f.h2;
    p.p3 = f.p3;
    p.stages = stages;
    p.slot_bytes = slot;
    p.err = f.conv[0].err;
    p.bar = f.bar;
    p.budget_ns = barrier_timeout_ns();
    // at least 120 KB: one CTA per SM, so that its 512-column TMEM
    // allocation never waits for another CTA's
    const size_t smem = std::max<size_t>(uf_smem_bytes(stages, slot), 120 * 1024);
    static std::once_flag once[64];
    static cudaError_t attr_err[64];
    std::call_once(once[di.device & 63], [&] {
        attr_err[di.device & 63] =
            cudaFuncSetAttribute(unet_fused_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM_MAX);
    });
    CFM_CUDA_TRY(attr_err[di.device & 63]);
    int per_sm = 0;
    CFM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, unet_fused_fwd, UF_THREADS, smem));
    if (per_sm != 1) {
        set_error("persistent U-Net forward: %d CTAs per SM (needs exactly one)", per_sm);
        return CFM_UNSUPPORTED;
    }
    void *args[] = {(void *)&m, (void *)&p};
    CFM_CUDA_TRY(launch_cooperative((const void *)unet_fused_fwd, dim3(di.num_sms), dim3(UF_THREADS), args, smem, s));
    return CFM_OK;
}

namespace {

// K splits of a weight gradient: at most two tiles per SM (so that no CTA
// runs a tile more than the others), each split at least four K steps.
long long wgrad_ksplit(int B, int H, int W, int Cin, int num_sms) {
    const int kc = W % 64 == 0 ? 64 : 32;
    const int ci_rows = std::min(Cin, 128);
    const int taps_per_tile = 128 / ci_rows;
    const long long base =
        (long long)((9 + taps_per_tile - 1) / taps_per_tile) * ((Cin + ci_rows - 1) / ci_rows);
    const long long total_k = (long long)B * H * (W / kc);
    long long ks = 2LL * num_sms / base;
    return std::max(1LL, std::min(ks, total_k / 4 > 0 ? total_k / 4 : 1));
}

}  // namespace

long long tc_wgrad_ws_floats(int B, int H, int W, int Cin, int Cout, int num_sms) {
    return wgrad_ksplit(B, H, W, Cin, num_sms) * 9LL * Cin * Cout;
}

int tc_conv_wgrad(const WgradArgs &a, cudaStream_t s) {
    CFM_ARG_CHECK(a.Cin % 32 == 0 && a.Cin <= 256, "Cin must be a multiple of 32, at most 256");
    CFM_ARG_CHECK(a.Cout == 32 || a.Cout == 64 || a.Cout == 128 || a.Cout == 256, "Cout");
    CFM_ARG_CHECK(a.W % 32 == 0, "W must be a multiple of 32");
    const long long per_split = 9LL * a.Cin * a.Cout;
    CFM_ARG_CHECK(a.ws && a.ws_floats >= per_split, "weight-gradient workspace too small");
    const int kc = a.W % 64 == 0 ? 64 : 32;
    TcConvParams p{};
    p.mode = 1;
    p.csplit = 1;
    p.B = a.B;
    p.H = a.H;
    p.W = a.W;
    p.Cin = a.Cin;
    p.Cout = a.Cout;
    p.ci_rows = std::min(a.Cin, 128);
    p.ci_tiles = (a.Cin + p.ci_rows - 1) / p.ci_rows;  // a partial last tile reads zero fill
    p.taps_per_tile = 128 / p.ci_rows;
    p.tap_groups = (9 + p.taps_per_tile - 1) / p.taps_per_tile;
    p.total_k = (long long)a.B * a.H * (a.W / kc);
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    const long long base = (long long)p.tap_groups * p.ci_tiles;
    const long long ks = std::min(wgrad_ksplit(a.B, a.H, a.W, a.Cin, di.num_sms), a.ws_floats / per_split);
    p.ksplit = (int)ks;
    p.ntiles = (int)(base * ks);
    p.dw = a.dw;
    p.wpart = a.ws;
    p.err = a.err;
    p.budget_ns = barrier_timeout_ns();
    p.a_cb = a.Cin % 64 == 0 ? 64 : 32;  // divides ci_rows
    p.b_cb = std::min(a.Cout, 64);
    // NHWC maps; a box is a_cb (b_cb) channels of KC pixels of one row
    CUtensorMap mx, mz;
    const cuuint64_t da[4] = {(cuuint64_t)a.Cin, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
    const cuuint64_t sa[3] = {(cuuint64_t)a.Cin * 2, (cuuint64_t)a.W * a.Cin * 2,
                              (cuuint64_t)a.H * a.W * a.Cin * 2};
    const cuuint32_t ba[4] = {(cuuint32_t)p.a_cb, (cuuint32_t)kc, 1, 1};
    if ((st = encode_map(&mx, a.x, 4, da, sa, ba, p.a_cb * 2))) return st;
    const cuuint64_t db[4] = {(cuuint64_t)a.Cout, (cuuint64_t)a.W, (cuuint64_t)a.H, (cuuint64_t)a.B};
    const cuuint64_t sb[3] = {(cuuint64_t)a.Cout * 2, (cuuint64_t)a.W * a.Cout * 2,
                              (cuuint64_t)a.H * a.W * a.Cout * 2};
    const cuuint32_t bb[4] = {(cuuint32_t)p.b_cb, (cuuint32_t)kc, 1, 1};
    if ((st = encode_map(&mz, a.dz, 4, db, sb, bb, p.b_cb * 2))) return st;
    if ((st = launch(kc, a.Cout, mx, mx, mz, p, s))) return st;
    const int blocks = (int)((per_split + WR_ENTRIES - 1) / WR_ENTRIES);
    CFM_CUDA_TRY(launch_pdl(tc_wgrad_reduce, dim3(blocks), dim3(WR_ENTRIES * WR_CHUNKS), 0, s,
                            (const float *)a.ws, p.ksplit, a.Cin, a.Cout, a.dw));
    return CFM_OK;
}

}  // namespace cfm

using namespace cfm;

namespace {

// Device scratch for the host-buffer entry points (freed on every path).
struct DevBufs {
    std::vector<void *> ptrs;
    ~DevBufs() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T **out, size_t count) {
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(p);
        *out = static_cast<T *>(p);
        return e;
    }
};

int finish_err(const int *err_dev) {
    int herr = 0;
    CFM_CUDA_TRY(cudaMemcpy(&herr, err_dev, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) {
        set_error("tensor-core convolution: a pipeline wait timed out (site %d)", herr);
        return CFM_BARRIER_TIMEOUT;
    }
    return CFM_OK;
}

}  // namespace

extern "C" {

int cfm_tc_conv3x3(int B, int H, int W, int Cin, int Cout, const unsigned short *x,
                   const unsigned short *w, const float *bias, int relu, unsigned short *out) {
    clear_error();
    CFM_ARG_CHECK(x && w && out, "null argument");
    CFM_ARG_CHECK(B >= 1 && H >= 1 && W >= 1, "sizes");
    const size_t nx = (size_t)B * H * W * Cin, no = (size_t)B * H * W * Cout,
                 nw = (size_t)9 * Cout * Cin;
    DevBufs d;
    __nv_bfloat16 *dx, *dw, *dout;
    float *db = nullptr;
    int *derr;
    CFM_CUDA_TRY(d.get(&dx, nx));
    CFM_CUDA_TRY(d.get(&dw, nw));
    CFM_CUDA_TRY(d.get(&dout, no));
    CFM_CUDA_TRY(d.get(&derr, 1));
    if (bias) CFM_CUDA_TRY(d.get(&db, Cout));
    CFM_CUDA_TRY(cudaMemcpy(dx, x, nx * 2, cudaMemcpyHostToDevice));
    CFM_CUDA_TRY(cudaMemcpy(dw, w, nw * 2, cudaMemcpyHostToDevice));
    if (bias) CFM_CUDA_TRY(cudaMemcpy(db, bias, Cout * 4, cudaMemcpyHostToDevice));
    CFM_CUDA_TRY(cudaMemset(derr, 0, sizeof(int)));
    float *dws;
    CFM_CUDA_TRY(d.get(&dws, (size_t)TC_WS_FLOATS));
    ConvArgs a{dx, dw, db, nullptr, dout, derr, B, H, W, Cin, Cout, relu};
    a.ws = dws;
    a.ws_floats = TC_WS_FLOATS;
    int st = tc_conv_fwd(a, 0);
    if (st) return st;
    CFM_CUDA_TRY(cudaDeviceSynchronize());
    if ((st = finish_err(derr))) return st;
    CFM_CUDA_TRY(cudaMemcpy(out, dout, no * 2, cudaMemcpyDeviceToHost));
    return CFM_OK;
}

int cfm_tc_conv3x3_wgrad(int B, int H, int W, int Cin, int Cout, const unsigned short *x,
                         const unsigned short *dz, float *dw_out) {
    clear_error();
    CFM_ARG_CHECK(x && dz && dw_out, "null argument");
    CFM_ARG_CHECK(B >= 1 && H >= 1 && W >= 1, "sizes");
    CFM_ARG_CHECK(Cin % 32 == 0 && Cin <= 256 && Cout % 32 == 0 && Cout <= 256, "channels");
    const size_t nx = (size_t)B * H * W * Cin, nz = (size_t)B * H * W * Cout,
                 nw = (size_t)9 * Cout * Cin;
    DevBufs d;
    __nv_bfloat16 *dx, *ddz;
    float *ddw;
    int *derr;
    CFM_CUDA_TRY(d.get(&dx, nx));
    CFM_CUDA_TRY(d.get(&ddz, nz));
    CFM_CUDA_TRY(d.get(&ddw, nw));
    CFM_CUDA_TRY(d.get(&derr, 1));
    CFM_CUDA_TRY(cudaMemcpy(dx, x, nx * 2, cudaMemcpyHostToDevice));
    CFM_CUDA_TRY(cudaMemcpy(ddz, dz, nz * 2, cudaMemcpyHostToDevice));
    CFM_CUDA_TRY(cudaMemset(ddw, 0, nw * 4));
    CFM_CUDA_TRY(cudaMemset(derr, 0, sizeof(int)));
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    const long long wsn = tc_wgrad_ws_floats(B, H, W, Cin, Cout, di.num_sms);
    float *dws;
    CFM_CUDA_TRY(d.get(&dws, (size_t)wsn));
    WgradArgs a{dx, ddz, ddw, derr, B, H, W, Cin, Cout, dws, wsn};
    if ((st = tc_conv_wgrad(a, 0))) return st;
    CFM_CUDA_TRY(cudaDeviceSynchronize());
    if ((st = finish_err(derr))) return st;
    CFM_CUDA_TRY(cudaMemcpy(dw_out, ddw, nw * 4, cudaMemcpyDeviceToHost));
    return CFM_OK;
}

}  // extern "C"
