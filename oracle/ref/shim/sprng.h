/* Stand-in for the SIMPLE_SPRNG interface that the reference's random_hao
 * uses (common/randomHao/source/random_hao.cpp): one stream per process,
 * the counter-based SplitMix64 stream of the engine and the oracle (uniform
 * k of seed s = mix(mix(s) + (k+1) * golden) >> 11, times 2^-53), so the
 * reference program draws exactly the numbers the engine draws.  Its packed
 * state is (seed, counter).  Oracle reference build only. */
#ifndef OR_SPRNG_SHIM_H
#define OR_SPRNG_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
#define SPRNG_DEFAULT 0
#define MAX_PACKED_LENGTH 64
int init_sprng(int gtype, int seed, int param);
int make_sprng_seed(void);
double sprng(void);
int pack_sprng(char **buffer);
int unpack_sprng(char *buffer);
#ifdef __cplusplus
}
#endif
#endif
