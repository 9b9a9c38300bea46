/* SplitMix64 stream behind the SPRNG stand-in (see sprng.h). */
#include "sprng.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t g_seed = 985456376u, g_counter = 0;

static uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int init_sprng(int gtype, int seed, int param)
{
    (void)gtype; (void)param;
    g_seed = (uint64_t)(int64_t)seed;
    g_counter = 0;
    return 0;
}

int make_sprng_seed(void) { return 985456376; }

double sprng(void)
{
    uint64_t b = mix64(mix64(g_seed) + (g_counter + 1ULL) * 0x9E3779B97F4A7C15ULL);
    g_counter++;
    return (double)(b >> 11) * (1.0 / 9007199254740992.0);
}

int pack_sprng(char **buffer)
{
    *buffer = (char *)malloc(16);
    memcpy(*buffer, &g_seed, 8);
    memcpy(*buffer + 8, &g_counter, 8);
    return 16;
}

int unpack_sprng(char *buffer)
{
    memcpy(&g_seed, buffer, 8);
    memcpy(&g_counter, buffer + 8, 8);
    return 0;
}
