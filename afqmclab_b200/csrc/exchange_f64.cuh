// FP64 exchange of the phaseless mixed estimator as dense GEMMs (real A);
// see exchange_f64.cu.
#pragma once
#include "common.cuh"
#include "walker_kernels.cuh"

struct afqmc_engine;

// Per spin block: X (K x G, the block's real A_g as columns) and V (K x K).
struct ExF64 {
    int b = 0, Ns = 0;
    long long K = 0;
    double *X = nullptr, *V = nullptr;
};

// The FP64 form's closed-shell and GEMM-exchange state: per-block operands,
// shared scratch (Z: K x W, M and R: K x K, Y: K x G) and the per-walker
// exchange totals; `restricted` when both spin blocks carry the same trial
// bit for bit (bl1 lists block 0 with multiplicity 2).
struct ExF64Scratch {
    zd *Z = nullptr, *M = nullptr, *R = nullptr, *Y = nullptr, *exTot = nullptr;
    // the force's K split: xsplit partial products (G x W each) in xp
    zd *xp = nullptr;
    int xsplit = 1;
    ExF64 blk[2];
    bool gemm = false, restricted = false;
    Blocks bl1{};
};

int exf64_alloc(afqmc_engine *e, long long Kmax, ExF64Scratch &s);
int exf64_build(afqmc_engine *e, int b, ExF64 &x);
// Adds block x's exchange: exTot[w] (+)= mult u^T V u, exNum[g] += mult x_g^T R x_g.
int exf64_run(afqmc_engine *e, const ExF64 &x, bool accumulate, int mult);
// The operands of spin block b (block 0's X and V when restricted, which are
// block 1's too: both blocks carry the same trial).
ExF64 exf64_block(const afqmc_engine *e, int b);
// Z = V U (Z(b + Ns i, w) = sum_g (D_gw A_g)(b, i)) and exTot[w] (+)= mult u_w^T Z_w.
int exf64_walker_totals(afqmc_engine *e, const ExF64 &x, bool accumulate, int mult);
// M = Uden Um^T (K x K) and its exchange permutation R, R(a + Ns i, b + Ns j) =
// M(b + Ns i, a + Ns j); Uden, Um are K x W with leading dimension K.
int exf64_pair_matrix(afqmc_engine *e, const ExF64 &x, const zd *Uden, const zd *Um);
// Force xbar(g, w) = mult sum_b x_g^T u_w over the blocks of bl, on the real X.
int exf64_force(afqmc_engine *e, const Blocks &bl);
