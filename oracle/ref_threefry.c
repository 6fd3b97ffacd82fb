/*
 * ref_threefry.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Exposes the reference's vendored Random123 generator
 * (external/include/Random123/threefry.h, u01.h), compiled where it lies, so
 * the restated generator and the device code can be pinned against it.
 * Built by oracle/build.py into oracle/_ref/libref_threefry.so.
 */
#define R123_USE_U01_DOUBLE 1
#include <Random123/threefry.h>
#include <Random123/u01.h>

void ref_threefry2x64(const unsigned long long ctr[2], const unsigned long long key[2], unsigned long long out[2])
{
    threefry2x64_ctr_t c = {{ctr[0], ctr[1]}};
    threefry2x64_key_t k = {{key[0], key[1]}};
    threefry2x64_ctr_t r = threefry2x64(c, k);
    out[0] = r.v[0];
    out[1] = r.v[1];
}

double ref_u01_open_open_64_53(unsigned long long w) { return u01_open_open_64_53(w); }
