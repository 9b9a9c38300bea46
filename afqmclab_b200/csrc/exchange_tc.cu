// Exchange term of the phaseless mixed estimator on the tcgen05 tensor cores
// (RealMaterialMoleculeMeasureFixedSD2sSD2is::calculateCholeskyEx, :258-284):
//   D_{g,w} = A_g theta_w  (Ns x Ns, complex),  ex[g, w] += sum_ab D_ab D_ba
// for one spin block per launch.  When every A_g is real (real trial and real
// Cholesky vectors, the molecular case) the imaginary-A products are skipped:
// D = A_re theta_re + i A_re theta_im, half the tensor work.  As a GEMM: rows (g, a) of A (K = orbital
// i), columns (w, b) of theta (K = i), both bf16 K-major; the 128 x 128 output
// tile holds 128/Ns vectors g times 128/Ns walkers w, and the epilogue reduces
// each Ns x Ns block to its trace tr(D D) without writing D.
//
// Persistent, warp-specialised: warp 0 TMA producer, warp 1 UMMA issuer (and
// TMEM owner, 512 columns = two accumulator pairs so the epilogue of one tile
// overlaps the MMAs of the next), warps 2..9 epilogue (two warps per TMEM lane
// quarter, each taking half of the columns).  The epilogue keeps each thread's
// row of a block in registers and reads the transposed entries from a
// swizzled shared-memory copy (bf16 pairs), so tr(D D) costs one shared
// store and one load per complex product.  A CTA takes a work item = one A tile (kept in shared
// memory) x a chunk of walker tiles.  All waits are bounded.
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>

#include "engine_internal.cuh"
#include "mixed.cuh"
#include "tc_common.cuh"
#include "tc_gemm.cuh"
#include "once.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

constexpr int XS_STAGES = 3;          // B stages: one 64-wide K box, both planes
constexpr int XS_NCHUNK = 32;         // walker tiles per work item
constexpr int XS_TILE_BYTES = 16384;  // 128 rows x 128 B

constexpr int XS_THREADS = 320;
constexpr int XS_EPI_WARPS = 8;

struct XSmem {
    // sA: 2 planes x 2 K boxes; sB: XS_STAGES x (2 planes); transpose: 8 warps x 32x32 float2
    static constexpr size_t bytes()
    {
        return 1024 + 4 * XS_TILE_BYTES + (size_t)XS_STAGES * 2 * XS_TILE_BYTES + XS_EPI_WARPS * 32 * 32 * 8 + 256;
    }
};

// swizzled 32 x 32 tile of 4-byte pairs (128-byte rows): element (r, c) at
// r * 32 + 4 * ((c / 4) ^ (r % 8)) + c % 4, so a row is written with
// 16-byte stores and a column is read without bank conflicts
__device__ __forceinline__ int tsw16(int r, int c) { return r * 32 + ((((c >> 2) ^ (r & 7)) << 2) | (c & 3)); }
// (re, im) as a bf16 pair: re in the low half, im in the high half
__device__ __forceinline__ uint32_t bf2bits(float re, float im)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(re, im);
    return *(const uint32_t *)&h;
}

template <int NS, bool REALA>
__global__ void __launch_bounds__(XS_THREADS, 1)
exchange_tc_kernel(const __grid_constant__ CUtensorMap tmAr, const __grid_constant__ CUtensorMap tmAi,
                   const __grid_constant__ CUtensorMap tmBr, const __grid_constant__ CUtensorMap tmBi,
                   int G, int W, int Ns, int n, const int *alive, zd *ex, int *err)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = base;                                   // [plane][kb] tiles
    uint8_t *sB = base + 4 * XS_TILE_BYTES;               // [stage][plane] tiles
    float2 *sT = (float2 *)(sB + (size_t)XS_STAGES * 2 * XS_TILE_BYTES);
    uint64_t *bars = (uint64_t *)(sT + XS_EPI_WARPS * 32 * 32);
    uint64_t *full = bars, *empty = bars + XS_STAGES;
    uint64_t *aFull = bars + 2 * XS_STAGES, *aEmpty = aFull + 1;
    uint64_t *accFull = aEmpty + 1, *accEmpty = accFull + 2;
    uint32_t *tslot = (uint32_t *)(accEmpty + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    (void)Ns;
    const int rowsTotal = G * NS;
    const int MT = (rowsTotal + 127) / 128;
    const int WB = 128 / NS;                      // walkers per tile
    const int NT = (W + WB - 1) / WB;             // walker tiles
    const int NCH = (NT + XS_NCHUNK - 1) / XS_NCHUNK;
    const int items = MT * NCH;
    const int KB = n / 64;

    if (threadIdx.x == 0) {
        for (int s = 0; s < XS_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(aFull, 1);
        mbar_init(aEmpty, 1);
        for (int b = 0; b < 2; ++b) { mbar_init(&accFull[b], 1); mbar_init(&accEmpty[b], XS_EPI_WARPS); }
        fence_mbar_init();
        tma_prefetch_desc(&tmAr); tma_prefetch_desc(&tmAi);
        tma_prefetch_desc(&tmBr); tma_prefetch_desc(&tmBi);
    }
    if (warp == 1) { tmem_alloc(tslot, 512); tmem_relinquish(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0, sphase = 0, itemCount = 0;
            for (int it = blockIdx.x; it < items && ok; it += gridDim.x, ++itemCount) {
                const int mt = it % MT, ch = it / MT;
                if (itemCount > 0) ok = mbar_wait(aEmpty, (itemCount - 1) & 1);
                if (!ok) break;
                mbar_arrive_expect_tx(aFull, (REALA ? 1 : 2) * KB * XS_TILE_BYTES);
                for (int kb = 0; kb < KB; ++kb) {
                    tma_load_2d(sA + (0 * 2 + kb) * XS_TILE_BYTES, &tmAr, aFull, kb * 64, mt * 128);
                    if (!REALA) tma_load_2d(sA + (1 * 2 + kb) * XS_TILE_BYTES, &tmAi, aFull, kb * 64, mt * 128);
                }
                const int t0 = ch * XS_NCHUNK, t1 = min(NT, t0 + XS_NCHUNK);
                for (int t = t0; t < t1 && ok; ++t) {
                    for (int kb = 0; kb < KB && ok; ++kb) {
                        ok = mbar_wait(&empty[stage], sphase ^ 1);
                        if (!ok) break;
                        mbar_arrive_expect_tx(&full[stage], 2 * XS_TILE_BYTES);
                        tma_load_3d(sB + (stage * 2 + 0) * XS_TILE_BYTES, &tmBr, &full[stage], kb * 64, 0, t * WB);
                        tma_load_3d(sB + (stage * 2 + 1) * XS_TILE_BYTES, &tmBi, &full[stage], kb * 64, 0, t * WB);
                        if (++stage == XS_STAGES) { stage = 0; sphase ^= 1; }
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t ID = idesc_bf16(128, 128), IDN = idesc_bf16(128, 128, true);
            int stage = 0, sphase = 0, itemCount = 0, tileCount = 0;
            for (int it = blockIdx.x; it < items && ok; it += gridDim.x, ++itemCount) {
                const int ch = it / MT;
                ok = mbar_wait(aFull, itemCount & 1);
                if (!ok) break;
                const int t0 = ch * XS_NCHUNK, t1 = min(NT, t0 + XS_NCHUNK);
                for (int t = t0; t < t1 && ok; ++t, ++tileCount) {
                    const int ab = tileCount & 1;
                    if (tileCount >= 2) ok = mbar_wait(&accEmpty[ab], ((tileCount >> 1) - 1) & 1);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t dR = tmem + ab * 256, dI = tmem + ab * 256 + 128;
                    for (int kb = 0; kb < KB && ok; ++kb) {
                        ok = mbar_wait(&full[stage], sphase);
                        if (!ok) break;
                        tc_fence_after();
                        const uint32_t ar = smem_u32(sA + (0 * 2 + kb) * XS_TILE_BYTES);
                        const uint32_t ai = smem_u32(sA + (1 * 2 + kb) * XS_TILE_BYTES);
                        const uint32_t br = smem_u32(sB + (stage * 2 + 0) * XS_TILE_BYTES);
                        const uint32_t bi = smem_u32(sB + (stage * 2 + 1) * XS_TILE_BYTES);
#pragma unroll
                        for (int kk = 0; kk < 4; ++kk) {
                            const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                            const uint64_t dar = desc_k_sw128(ar + kk * 32), dai = desc_k_sw128(ai + kk * 32);
                            const uint64_t dbr = desc_k_sw128(br + kk * 32), dbi = desc_k_sw128(bi + kk * 32);
                            umma_bf16(dR, dar, dbr, ID, acc);
                            umma_bf16(dI, dar, dbi, ID, acc);
                            if (!REALA) {
                                umma_bf16(dR, dai, dbi, IDN, 1u);
                                umma_bf16(dI, dai, dbr, ID, 1u);
                            }
                        }
                        umma_commit(&empty[stage]);
                        if (++stage == XS_STAGES) { stage = 0; sphase ^= 1; }
                    }
                    umma_commit(&accFull[ab]);
                }
                umma_commit(aEmpty);
            }
        }
        __syncwarp();
    } else {
        const int q = warp & 3, half = (warp - 2) >> 2;
        float2 *T = sT + (warp - 2) * 32 * 32;
        const int r = q * 32 + lane;                   // tile row = (g_local, a)
        const int a = r % NS;
        const int gl = r / NS;                         // g inside the tile
        const int rb = lane - a;                       // first warp row of this thread's g
        int tileCount = 0;
        for (int it = blockIdx.x; it < items && ok; it += gridDim.x) {
            const int mt = it % MT, ch = it / MT;
            const int t0 = ch * XS_NCHUNK, t1 = min(NT, t0 + XS_NCHUNK);
            const int gg = mt * (128 / NS) + gl;
            for (int t = t0; t < t1 && ok; ++t, ++tileCount) {
                const int ab = tileCount & 1;
                ok = mbar_wait(&accFull[ab], (tileCount >> 1) & 1);
                if (!ok) break;
                tc_fence_after();
                const uint32_t tR = tmem + ab * 256 + ((uint32_t)(q * 32) << 16);
                const uint32_t tI = tR + 128;
#pragma unroll 1
                for (int c0 = half * 64; c0 < half * 64 + 64; c0 += 32) {
                    float vr[32], vi[32];
                    {
                        uint32_t ur[32], ui[32];
                        tmem_ld32_nw(tR + c0, ur);
                        tmem_ld32_nw(tI + c0, ui);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 32; ++j) { vr[j] = __uint_as_float(ur[j]); vi[j] = __uint_as_float(ui[j]); }
                    }
                    // The transposed factor goes through shared memory as bf16
                    // pairs (half the bytes of fp32, fp32's range); the register
                    // factor and the accumulation stay fp32.
                    float2 acc[32 / NS];
                    {
                        uint32_t *T16 = (uint32_t *)T;
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            uint4 pk;
                            pk.x = bf2bits(vr[j], vi[j]);
                            pk.y = bf2bits(vr[j + 1], vi[j + 1]);
                            pk.z = bf2bits(vr[j + 2], vi[j + 2]);
                            pk.w = bf2bits(vr[j + 3], vi[j + 3]);
                            *(uint4 *)(T16 + tsw16(lane, j)) = pk;
                        }
                        __syncwarp();
#pragma unroll
                        for (int wb = 0; wb < 32 / NS; ++wb) {
                            float sr0 = 0.f, si0 = 0.f, sr1 = 0.f, si1 = 0.f;
#pragma unroll
                            for (int b = 0; b < NS; ++b) {
                                const float xr = vr[wb * NS + b], xi = vi[wb * NS + b];
                                const uint32_t u = T16[tsw16(rb + b, wb * NS + a)];
                                const float yx = __uint_as_float(u << 16), yy = __uint_as_float(u & 0xffff0000u);
                                if (b & 1) { sr1 += xr * yx - xi * yy; si1 += xr * yy + xi * yx; }
                                else { sr0 += xr * yx - xi * yy; si0 += xr * yy + xi * yx; }
                            }
                            acc[wb] = make_float2(sr0 + sr1, si0 + si1);
                        }
                    }
                    // blocks (g, walker) of this 32-column chunk: D[a][b] in
                    // registers, D[b][a] from the transposed copy; reduce over a
#pragma unroll
                    for (int wb = 0; wb < 32 / NS; ++wb) {
                        float sr = acc[wb].x, si = acc[wb].y;
#pragma unroll
                        for (int o = NS >> 1; o > 0; o >>= 1) {
                            sr += __shfl_xor_sync(0xffffffffu, sr, o);
                            si += __shfl_xor_sync(0xffffffffu, si, o);
                        }
                        const int w = t * WB + (c0 + wb * NS) / NS;
                        if (a == 0 && gg < G && w < W) ex[gg + (size_t)G * w] = make_double2(sr, si);
                    }
                    __syncwarp();
                }
                tc_fence_before();
                if (lane == 0) mbar_arrive(&accEmpty[ab]);
            }
        }
    }
    if (!ok && err) atomicExch(err, 3);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1) tmem_dealloc(tmem, 512);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// theta of spin block b for every walker: dims {n (i), Ns (b), W (w)}
int make_map_theta(CUtensorMap *map, const void *base, int n, int Ns, int W, long long walkerPitch)
{
    auto enc = encode_fn();
    if (!enc) return -1;
    cuuint64_t dims[3] = {(cuuint64_t)n, (cuuint64_t)Ns, (cuuint64_t)W};
    cuuint64_t strides[2] = {(cuuint64_t)n * 2, (cuuint64_t)walkerPitch * 2};
    cuuint32_t box[3] = {64u, (cuuint32_t)Ns, (cuuint32_t)(128 / Ns)};
    cuuint32_t estr[3] = {1u, 1u, 1u};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void *>(base), dims, strides, box,
                     estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? 0 : (int)r + 10000;
}

template <int NS, bool REALA>
void launch_ns_a(int grid, size_t smem, cudaStream_t s, const CUtensorMap &ar, const CUtensorMap &ai,
                 const CUtensorMap &br, const CUtensorMap &bi, int G, int W, int n, const int *alive, zd *ex,
                 int *err)
{
    static std::atomic<unsigned long long> attr{0};
    if (first_on_device(attr)) {
        cudaFuncSetAttribute(exchange_tc_kernel<NS, REALA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
    exchange_tc_kernel<NS, REALA><<<grid, XS_THREADS, smem, s>>>(ar, ai, br, bi, G, W, NS, n, alive, ex, err);
}

template <int NS>
void launch_ns(bool realA, int grid, size_t smem, cudaStream_t s, const CUtensorMap &ar, const CUtensorMap &ai,
               const CUtensorMap &br, const CUtensorMap &bi, int G, int W, int n, const int *alive, zd *ex,
               int *err)
{
    if (realA) launch_ns_a<NS, true>(grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err);
    else launch_ns_a<NS, false>(grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err);
}

}  // namespace

// A2 operand of spin block b: rows (g, a) -> r = g Ns + a, K = i; two bf16 planes
__global__ void build_a2_kernel(int G, int Ns, int n, long long Ktot, long long tOff, const zd *Aall,
                                __nv_bfloat16 *A2r, __nv_bfloat16 *A2i)
{
    const long long total = (long long)G * Ns * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        long long r = e / n;
        int i = (int)(e % n);
        int g = (int)(r / Ns), a = (int)(r % Ns);
        zd v = Aall[(size_t)g * Ktot + tOff + a + (size_t)Ns * i];
        A2r[e] = __double2bfloat16(v.x);
        A2i[e] = __double2bfloat16(v.y);
    }
}

int exchange_tc_supported(int n, int Ns) { return (n == 64 || n == 128) && Ns > 0 && 32 % Ns == 0; }

// ex (G x W, complex) = exchange of one spin block (every (g, w) written once)
int exchange_tc_launch(cudaStream_t s, int G, int W, int Ns, int n, const __nv_bfloat16 *A2r,
                       const __nv_bfloat16 *A2i, const __nv_bfloat16 *Theta, long long tOff,
                       long long Ktot, const int *alive, zd *ex, int *err, bool realA)
{
    g_launch_count++;
    CUtensorMap ar, ai, br, bi;
    int r = tc_make_map_bf16(&ar, A2r, n, (long long)G * Ns, n, 128);
    if (!r) r = tc_make_map_bf16(&ai, A2i, n, (long long)G * Ns, n, 128);
    if (!r) r = make_map_theta(&br, Theta + tOff, n, Ns, W, 2 * Ktot);
    if (!r) r = make_map_theta(&bi, Theta + Ktot + tOff, n, Ns, W, 2 * Ktot);
    if (r) return r;
    const size_t smem = XSmem::bytes();
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int MT = (G * Ns + 127) / 128;
    const int NT = (W + 128 / Ns - 1) / (128 / Ns);
    const int items = MT * ((NT + XS_NCHUNK - 1) / XS_NCHUNK);
    const int grid = std::min(items, sms);
    switch (Ns) {
    case 1: launch_ns<1>(realA, grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err); break;
    case 2: launch_ns<2>(realA, grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err); break;
    case 4: launch_ns<4>(realA, grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err); break;
    case 8: launch_ns<8>(realA, grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err); break;
    case 16: launch_ns<16>(realA, grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err); break;
    default: launch_ns<32>(realA, grid, smem, s, ar, ai, br, bi, G, W, n, alive, ex, err); break;
    }
    return (int)cudaGetLastError();
}
