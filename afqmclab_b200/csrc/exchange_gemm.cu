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
// 32 x 32 tiles (q, w) through shared memory.
__global__ void __launch_bounds__(256)
ex_transpose_kernel(int W, long long K, long long Ktot, long long tOff, const __nv_bfloat16 *Theta,
                    const zd *logov, const int *alive, const double *shift, __nv_bfloat16 *Bt,
                    __nv_bfloat16 *Ar, __nv_bfloat16 *Ai)
{
    __shared__ float tr[32][33], ti[32][33];
    __shared__ double dr[32], di[32];
    const long long q0 = (long long)blockIdx.x * 32;
    const int w0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 8 rows of 32
    if (threadIdx.x < 32) {
        const int w = w0 + threadIdx.x;
        double r = 0.0, im = 0.0;
        if (w < W && alive[w]) {
            const zd d = zexp(make_double2(logov[w].x - shift[0], logov[w].y));
            r = d.x; im = d.y;
        }
        dr[threadIdx.x] = r; di[threadIdx.x] = im;
    }
    for (int r = ty; r < 32; r += 8) {
        const int w = w0 + r;
        const long long q = q0 + tx;
        float vr = 0.f, vi = 0.f;
        if (w < W && q < K) {
            const __nv_bfloat16 *t = Theta + (size_t)w * 2 * Ktot + tOff + q;
            vr = __bfloat162float(t[0]);
            vi = __bfloat162float(t[Ktot]);
        }
        tr[r][tx] = vr;
        ti[r][tx] = vi;
    }
    __syncthreads();
    const long long W2 = 2LL * W;
    for (int r = ty; r < 32; r += 8) {
        const long long q = q0 + r;
        const int w = w0 + tx;
        if (q >= K || w >= W) continue;
        const float ur = tr[tx][r], ui = ti[tx][r];
        const double vr = dr[tx] * ur - di[tx] * ui, vi = dr[tx] * ui + di[tx] * ur;
        Bt[q * W2 + w] = __float2bfloat16(ur);
        Bt[q * W2 + W + w] = __float2bfloat16(ui);
        Ar[q * W2 + w] = __double2bfloat16(vr);
        Ar[q * W2 + W + w] = __double2bfloat16(-vi);
        Ai[q * W2 + w] = __double2bfloat16(vi);
        Ai[q * W2 + W + w] = __double2bfloat16(vr);
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
        dim3 tg((unsigned)((K + 31) / 32), (unsigned)((W + 31) / 32));
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
