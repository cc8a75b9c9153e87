/* dropin_io.h -- deterministic inputs and a plain record file for the
 * drop-in programs: records of (16-byte name, int64 count, count doubles),
 * read back by tests/test_gpu_dropin.py. */
#ifndef TBLIS_B200_TEST_DROPIN_IO_H
#define TBLIS_B200_TEST_DROPIN_IO_H

#include <stdint.h>
#include <stdio.h>
#include <string.h>

/* splitmix64 -> uniform double in [-1, 1) */
static double dropin_uniform(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30))*0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27))*0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11)*(1.0/9007199254740992.0)*2.0 - 1.0;
}

static void dropin_fill(double* x, long n, uint64_t seed)
{
    for (long i = 0; i < n; i++) x[i] = dropin_uniform(&seed);
}

static void dropin_record(FILE* f, const char* name, const double* x, long n)
{
    char tag[16];
    memset(tag, 0, sizeof(tag));
    strncpy(tag, name, sizeof(tag) - 1);
    int64_t cnt = n;
    fwrite(tag, 1, sizeof(tag), f);
    fwrite(&cnt, sizeof(cnt), 1, f);
    fwrite(x, sizeof(double), (size_t)n, f);
}

#endif
