// Exchange term of the phaseless mixed estimator as dense GEMMs, for real
// half-rotated Cholesky vectors A_g (real trial, real L_g).  Per spin block
// (Ns electrons, n orbitals, K = Ns n) and walker w, with
// u_w(i + n b) = theta_w(i, b):
//
//   sum_g ex[g, w] = sum_g tr(D_gw D_gw) = u_w^T V u_w,
//       V(i + n b, j + n a) = sum_g A_g(a, i) A_g(b, j)    (K x K, symmetric,
//       built once in FP64 and rounded to bf16)
//   exNum[g] += sum_w den_w ex[g, w] = x_g^T R x_g,  x_g(i + n a) = A_g(a, i),
//       R(i + n a, j + n b) = M(i + n b, j + n a),  M = sum_w den_w u_w u_w^T
//
// calculateCholeskyEx (afqmc/model/realMaterialMolecule/source/
// realMaterialMoleculeMeasureFixedSD2sSD2is.cpp:258-284) computes ex[g, w] block by block; here the energy needs only its sum over g
// and the per-vector accumulator only its den-weighted sum over walkers, and
// both are quadratic forms evaluated with tensor-core GEMMs (tc_gemm_bf16):
//   Z = V U^T (K x 2W), ex_w = sum_q u_w(q) Z_w(q)           (energy)
//   M_re, M_im = [den u]^T-weighted outer products over walkers (K x K)
//   Y_g = [R_re | R_im]^T x_g (2K per vector), exNum_g = sum_q x_g(q) Y_g(q)
// For K = 4096, W = 2048, G = 640 this is about 0.23 T multiply-adds per spin
// instead of 0.34 T for the blockwise form, all in plain GEMMs.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <vector>

#include "engine_internal.cuh"
#include "exchange_gemm.cuh"
#include "tc_gemm.cuh"
#include "zgemm.cuh"

extern std::atomic<long long> g_launch_count;

namespace {

// V(q2, q1) from C = Aflat Aflat^T (K x K complex FP64, index c = a + Ns i,
// column-major): V(j + n a, i + n b) = C(a + Ns i, b + Ns j) (real part)
__global__ void vprime_kernel(int n, int Ns, const zd *C, __nv_bfloat16 *V)
{
    const long long K = (long long)n * Ns;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < K * K;
         e += (long long)gridDim.x * blockDim.x) {
        const long long q2 = e / K, q1 = e % K;
        const int j = (int)(q2 % n), a = (int)(q2 / n), i = (int)(q1 % n), b = (int)(q1 / n);
        const zd v = C[(size_t)(a + (long long)Ns * i) + (size_t)K * (b + (long long)Ns * j)];
        V[e] = __double2bfloat16(v.x);
    }
}

// shift[0] = max over alive walkers of Re logov (0 when none is alive): the
// walker factors exp(logov - shift) stay within the bf16 exponent range
__global__ void __launch_bounds__(256) ex_shift_kernel(int W, const zd *logov, const int *alive, double *shift)
{
    __shared__ double red[32];
    double m = -1e300;
    for (int w = threadIdx.x; w < W; w += blockDim.x)
        if (alive[w]) m = fmax(m, logov[w].x);
    m = block_max(m, red);
    if (threadIdx.x == 0) shift[0] = m > -1e299 ? m : 0.0;
}

// Operands of M over the walkers (K-major in the walker index, 2W per row):
//   Bt(q) = [u_re(q, .) | u_im(q, .)],  Ar(q) = [v_re | -v_im],  Ai(q) = [v_im | v_re],
// v_w = exp(logov_w - shift) u_w for alive walkers and 0 otherwise.
// 64 x 64 tiles (q, w) through shared memory; theta rows are read and the
// operand rows written 8 bf16 (16 bytes) at a time.
constexpr int EXT = 64;

__device__ __forceinline__ uint32_t bf2pack(float a, float b)
{
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *(const uint32_t *)&h;
}

__global__ void __launch_bounds__(256)
ex_transpose_kernel(int W, long long K, long long Ktot, long long tOff, const __nv_bfloat16 *Theta,
                    const zd *logov, const int *alive, const double *shift, __nv_bfloat16 *Bt,
                    __nv_bfloat16 *Ar, __nv_bfloat16 *Ai)
{
    __shared__ float tr[EXT][EXT + 1], ti[EXT][EXT + 1];   // [walker][q]
    __shared__ double dr[EXT], di[EXT];
    const long long q0 = (long long)blockIdx.x * EXT;
    const int w0 = blockIdx.y * EXT;
    const int tid = threadIdx.x;
    if (tid < EXT) {
        const int w = w0 + tid;
        double r = 0.0, im = 0.0;
        if (w < W && alive[w]) {
            const zd d = zexp(make_double2(logov[w].x - shift[0], logov[w].y));
            r = d.x; im = d.y;
        }
        dr[tid] = r; di[tid] = im;
    }
    // 64 walkers x 8 runs of 8 q per plane
    for (int idx = tid; idx < EXT * 8; idx += 256) {
        const int r = idx >> 3, c8 = (idx & 7) * 8;
        const int w = w0 + r;
        const long long q = q0 + c8;
        float vr[8], vi[8];
        if (w < W && q + 8 <= K) {
            const __nv_bfloat16 *t = Theta + (size_t)w * 2 * Ktot + tOff + q;
            const uint4 a = *(const uint4 *)t, b = *(const uint4 *)(t + Ktot);
            const uint32_t av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 fa = __bfloat1622float2(*(const __nv_bfloat162 *)&av[j]);
                const float2 fb = __bfloat1622float2(*(const __nv_bfloat162 *)&bv[j]);
                vr[2 * j] = fa.x; vr[2 * j + 1] = fa.y;
                vi[2 * j] = fb.x; vi[2 * j + 1] = fb.y;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const bool in = w < W && q + j < K;
                const __nv_bfloat16 *t = Theta + (size_t)(in ? w : 0) * 2 * Ktot + tOff + (in ? q + j : 0);
                vr[j] = in ? __bfloat162float(t[0]) : 0.f;
                vi[j] = in ? __bfloat162float(t[Ktot]) : 0.f;
            }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) { tr[r][c8 + j] = vr[j]; ti[r][c8 + j] = vi[j]; }
    }
    __syncthreads();
    const long long W2 = 2LL * W;
    // 64 q rows x 8 runs of 8 walkers; each run goes to six 16-byte pieces
    for (int idx = tid; idx < EXT * 8; idx += 256) {
        const int qr = idx >> 3, c8 = (idx & 7) * 8;
        const long long q = q0 + qr;
        const int wb = w0 + c8;
        if (q >= K || wb >= W) continue;
        float ur[8], ui[8], xr[8], xi[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            ur[j] = tr[c8 + j][qr];
            ui[j] = ti[c8 + j][qr];
            xr[j] = (float)(dr[c8 + j] * ur[j] - di[c8 + j] * ui[j]);
            xi[j] = (float)(dr[c8 + j] * ui[j] + di[c8 + j] * ur[j]);
        }
        const size_t row = (size_t)q * W2;
        if ((W & 7) == 0 && wb + 8 <= W) {
            uint4 a, b, c, d;
            a.x = bf2pack(ur[0], ur[1]); a.y = bf2pack(ur[2], ur[3]); a.z = bf2pack(ur[4], ur[5]); a.w = bf2pack(ur[6], ur[7]);
            b.x = bf2pack(ui[0], ui[1]); b.y = bf2pack(ui[2], ui[3]); b.z = bf2pack(ui[4], ui[5]); b.w = bf2pack(ui[6], ui[7]);
            c.x = bf2pack(xr[0], xr[1]); c.y = bf2pack(xr[2], xr[3]); c.z = bf2pack(xr[4], xr[5]); c.w = bf2pack(xr[6], xr[7]);
            d.x = bf2pack(xi[0], xi[1]); d.y = bf2pack(xi[2], xi[3]); d.z = bf2pack(xi[4], xi[5]); d.w = bf2pack(xi[6], xi[7]);
            uint4 nd;   // -v_im
            nd.x = d.x ^ 0x80008000u; nd.y = d.y ^ 0x80008000u; nd.z = d.z ^ 0x80008000u; nd.w = d.w ^ 0x80008000u;
            *(uint4 *)(Bt + row + wb) = a;
            *(uint4 *)(Bt + row + W + wb) = b;
            *(uint4 *)(Ar + row + wb) = c;
            *(uint4 *)(Ar + row + W + wb) = nd;
            *(uint4 *)(Ai + row + wb) = d;
            *(uint4 *)(Ai + row + W + wb) = c;
        } else {
            for (int j = 0; j < 8 && wb + j < W; ++j) {
                const int w = wb + j;
                Bt[row + w] = __float2bfloat16(ur[j]);
                Bt[row + W + w] = __float2bfloat16(ui[j]);
                Ar[row + w] = __float2bfloat16(xr[j]);
                Ar[row + W + w] = __float2bfloat16(-xi[j]);
                Ai[row + w] = __float2bfloat16(xi[j]);
                Ai[row + W + w] = __float2bfloat16(xr[j]);
            }
        }
    }
}

// exNum[g] += mult exp(shift) sum_q x_g(q) (Y_g(q) + i Y_g(K + q)), Y_g = row g (2K)
__global__ void __launch_bounds__(256)
ex_rowdot_kernel(long long K, const __nv_bfloat16 *X, const float *Y, const double *shift, double mult,
                 zd *exNum)
{
    __shared__ double red[32];
    const int g = blockIdx.x;
    const __nv_bfloat16 *x = X + (size_t)g * K;
    const float *y = Y + (size_t)g * 2 * K;
    double sr = 0.0, si = 0.0;
    for (long long q = threadIdx.x; q < K; q += blockDim.x) {
        const double xv = __bfloat162float(x[q]);
        sr += xv * y[q];
        si += xv * y[K + q];
    }
    sr = block_sum(sr, red);
    si = block_sum(si, red);
    if (threadIdx.x == 0) {
        const double f = mult * exp(shift[0]);
        exNum[g] = zadd(exNum[g], make_double2(f * sr, f * si));
    }
}

// exTot[w] (+)= mult sum_q u_w(q) (Z_w,re(q) + i Z_w,im(q)), Z column-major (ld K)
__global__ void __launch_bounds__(256)
ex_dot_kernel(int W, long long K, long long Ktot, long long tOff, const __nv_bfloat16 *Theta, const float *Z,
              int accumulate, double mult, zd *exTot)
{
    __shared__ double red[32];
    const int w = blockIdx.x;
    const __nv_bfloat16 *ur = Theta + (size_t)w * 2 * Ktot + tOff, *ui = ur + Ktot;
    const float *zr = Z + (size_t)K * (2 * w), *zi = zr + K;
    double sr = 0.0, si = 0.0;
    for (long long q = threadIdx.x; q < K; q += blockDim.x) {
        const double a = __bfloat162float(ur[q]), b = __bfloat162float(ui[q]);
        const double c = zr[q], d = zi[q];
        sr += a * c - b * d;
        si += a * d + b * c;
    }
    sr = block_sum(sr, red);
    si = block_sum(si, red);
    if (threadIdx.x == 0) {
        const zd v = make_double2(mult * sr, mult * si);
        exTot[w] = accumulate ? zadd(exTot[w], v) : v;
    }
}

}  // namespace

bool exchange_gemm_supported(int n, int Ns, int W, int G)
{
    // operand pitches (K, 2W, Ktot) and offsets 16-byte multiples for the TMA
    // maps; the exchanged store of M wants whole 32-orbital runs and K a
    // multiple of the 256-row tile; K x K scratch bounded to 2^28 elements
    const long long K = (long long)n * Ns;
    return Ns > 0 && n % 32 == 0 && K % 256 == 0 && W % 4 == 0 && G > 0 && K * K <= (1LL << 28);
}

int exchange_gemm_build(afqmc_engine *e, int b, ExGemmBlock &blk)
{
    const int n = e->n, Ns = e->bl.Ns[b], G = e->G;
    const long long K = (long long)n * Ns;
    blk.Ns = Ns;
    blk.K = K;
    blk.tOff = e->bl.tOff[b];
    // C = Aflat Aflat^T over the vectors, Aflat(c, g) = A_g(a, i), c = a + Ns i
    zd *C = nullptr;
    if (cudaMalloc(&C, sizeof(zd) * K * K) != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, "exchange setup: alloc");
    ZGemmArgs g;
    g.m = (int)K; g.n = (int)K; g.k = G;
    g.opA = OP_N; g.opB = OP_T;
    g.A = e->Aall + e->bl.tOff[b]; g.lda = e->Ktot;
    g.B = e->Aall + e->bl.tOff[b]; g.ldb = e->Ktot;
    g.C = C; g.ldc = K;
    cudaError_t ce = zgemm_batched(g, e->stream);
    if (ce != cudaSuccess) { cudaFree(C); return engine_fail(AFQMC_ERR_CUDA, "exchange setup: gemm"); }
    int r = engine_dalloc(e, (unsigned short **)&blk.V, (size_t)(K * K));
    if (r) { cudaFree(C); return r; }
    g_launch_count++;
    vprime_kernel<<<1184, 256, 0, e->stream>>>(n, Ns, C, blk.V);
    ce = cudaStreamSynchronize(e->stream);
    cudaFree(C);
    if (ce != cudaSuccess) return engine_fail(AFQMC_ERR_CUDA, "exchange setup");
    return engine_check_launch();
}

int exchange_gemm_alloc(afqmc_engine *e, long long Kmax, ExGemmScratch &s)
{
    const long long W2 = 2LL * e->W;
    int r = engine_dalloc(e, (unsigned short **)&s.Bt, (size_t)(Kmax * W2));
    if (!r) r = engine_dalloc(e, (unsigned short **)&s.Av, (size_t)(2 * Kmax * W2));
    if (!r) r = engine_dalloc(e, (unsigned short **)&s.Rt, (size_t)(2 * Kmax * Kmax));
    if (!r) r = engine_dalloc(e, &s.Y, (size_t)(e->G * 2 * Kmax));
    if (!r) r = engine_dalloc(e, &s.Z, (size_t)(Kmax * W2));
    if (!r) r = engine_dalloc(e, &s.shift, 1);
    return r;
}

int exchange_gemm_run(afqmc_engine *e, const ExGemmBlock &blk, const __nv_bfloat16 *A2r,
                      const __nv_bfloat16 *Theta, const ExGemmScratch &s, bool accumulate, int mult,
                      zd *exTot, zd *exNum, int *err)
{
    cudaStream_t st = e->stream;
    const int W = e->W, G = e->G, n = e->n;
    const long long K = blk.K, W2 = 2LL * W;
    // energy: Z = V U^T (column 2w + p = plane p of walker w), exTot_w (+)= u_w^T Z_w
    {
        TcGemmArgs a;
        a.M = (int)K; a.N = (int)W2; a.K = (int)K;
        a.A = blk.V; a.lda = K;
        a.B = Theta + blk.tOff; a.ldb = e->Ktot;
        a.C = s.Z; a.ldc = K; a.outType = TC_OUT_F32; a.err = err;
        int r = tc_gemm_bf16(a, st);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "exchange Z gemm: " + std::to_string(r));
        g_launch_count++;
        ex_dot_kernel<<<W, 256, 0, st>>>(W, K, e->Ktot, blk.tOff, Theta, s.Z, accumulate ? 1 : 0, (double)mult,
                                         exTot);
    }
    // per vector: M = sum_w den_w u_w u_w^T, Rt = M with b and a exchanged,
    // Y_g = Rt x_g, exNum_g += x_g^T Y_g
    {
        // the shift depends only on the walkers: once per measurement
        if (!accumulate) {
            g_launch_count++;
            ex_shift_kernel<<<1, 256, 0, st>>>(W, e->logov, e->alive, s.shift);
        }
        g_launch_count++;
        dim3 tg((unsigned)((K + EXT - 1) / EXT), (unsigned)((W + EXT - 1) / EXT));
        ex_transpose_kernel<<<tg, 256, 0, st>>>(W, K, e->Ktot, blk.tOff, Theta, e->logov, e->alive, s.shift,
                                                s.Bt, s.Av, s.Av + K * W2);
        // [M_re; M_im] = [Ar; Ai] Bt^T, stored exchanged as Rt
        TcGemmArgs a;
        a.M = (int)(2 * K); a.N = (int)K; a.K = (int)W2;
        a.A = s.Av; a.lda = W2;
        a.B = s.Bt; a.ldb = W2;
        a.C = s.Rt; a.outType = TC_OUT_BF16; a.err = err;
        a.permN = n; a.permK = K;
        int r = tc_gemm_bf16(a, st);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "exchange M gemm: " + std::to_string(r));
        TcGemmArgs y;
        y.M = (int)(2 * K); y.N = G; y.K = (int)K;
        y.A = s.Rt; y.lda = K;
        y.B = A2r; y.ldb = K;
        y.C = s.Y; y.ldc = 2 * K; y.outType = TC_OUT_F32; y.err = err;
        r = tc_gemm_bf16(y, st);
        if (r) return engine_fail(AFQMC_ERR_CUDA, "exchange Y gemm: " + std::to_string(r));
        g_launch_count++;
        ex_rowdot_kernel<<<G, 256, 0, st>>>(K, A2r, s.Y, s.shift, (double)mult, exNum);
    }
    return engine_check_launch();
}
