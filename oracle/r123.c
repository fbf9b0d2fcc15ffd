/* CPU restatement of chai's Random123 generators; see r123.h for the
 * reference lines each part follows.  Test infrastructure only. */
#include "r123.h"

#include <math.h>
#include <string.h>

/* ---------------------------------------------------------------- Philox */

static inline uint32_t mulhilo32(uint32_t a, uint32_t b, uint32_t* hi)
{
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
}

static inline uint64_t mulhilo64(uint64_t a, uint64_t b, uint64_t* hi)
{
    unsigned __int128 p = (unsigned __int128)a * (unsigned __int128)b;
    *hi = (uint64_t)(p >> 64);
    return (uint64_t)p;
}

/* R123Philox.cpp:117-211: one round; 4x32 multipliers D2511F53 / CD9E8D57 */
static void philox4x32_round(uint32_t c[4], const uint32_t k[2])
{
    uint32_t hi0, hi1;
    uint32_t lo0 = mulhilo32(0xD2511F53u, c[0], &hi0);
    uint32_t lo1 = mulhilo32(0xCD9E8D57u, c[2], &hi1);
    uint32_t o0 = hi1 ^ c[1] ^ k[0];
    uint32_t o2 = hi0 ^ c[3] ^ k[1];
    c[0] = o0; c[1] = lo1; c[2] = o2; c[3] = lo0;
}

void r123_philox4x32_R(unsigned R, const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    for (unsigned r = 0; r < R; r++) {
        if (r > 0) { k[0] += 0x9E3779B9u; k[1] += 0xBB67AE85u; }   /* bumpkey :63-115 */
        philox4x32_round(c, k);
    }
    memcpy(out, c, sizeof c);
}

void r123_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    r123_philox4x32_R(10, ctr, key, out);
}

void r123_philox2x32(const uint32_t ctr[2], const uint32_t key[1], uint32_t out[2])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], k = key[0];
    for (unsigned r = 0; r < 10; r++) {
        if (r > 0) k += 0x9E3779B9u;
        uint32_t hi;
        uint32_t lo = mulhilo32(0xd256d193u, c0, &hi);
        c0 = hi ^ k ^ c1;
        c1 = lo;
    }
    out[0] = c0; out[1] = c1;
}

void r123_philox2x64(const uint64_t ctr[2], const uint64_t key[1], uint64_t out[2])
{
    uint64_t c0 = ctr[0], c1 = ctr[1], k = key[0];
    for (unsigned r = 0; r < 10; r++) {
        if (r > 0) k += 0x9E3779B97F4A7C15ull;
        uint64_t hi;
        uint64_t lo = mulhilo64(0xD2B74407B1CE6E93ull, c0, &hi);
        c0 = hi ^ k ^ c1;
        c1 = lo;
    }
    out[0] = c0; out[1] = c1;
}

/* -------------------------------------------------------------- Threefry */

static inline uint32_t rotl32(uint32_t x, unsigned n) { n &= 31; return n ? (x << n) | (x >> (32 - n)) : x; }
static inline uint64_t rotl64(uint64_t x, unsigned n) { n &= 63; return n ? (x << n) | (x >> (64 - n)) : x; }

/* rotation tables, R123Threefry.cpp:50-112 */
static const unsigned ROT_32x4[8][2] = {{10, 26}, {11, 21}, {13, 27}, {23, 5},
                                        {6, 20}, {17, 11}, {25, 10}, {18, 20}};
static const unsigned ROT_32x2[8] = {13, 15, 26, 6, 17, 29, 16, 24};
static const unsigned ROT_64x2[8] = {16, 42, 12, 31, 16, 32, 24, 21};

/* Upstream Threefry4x32 (Random123/r123threefry.i:472-625): even rounds mix
 * lane pairs (0,1),(2,3), odd rounds (0,3),(2,1). */
void r123_threefry4x32_R(unsigned R, const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4])
{
    uint32_t ks[5], x[4];
    ks[4] = 0x1BD11BDAu;
    for (int i = 0; i < 4; i++) { ks[i] = key[i]; x[i] = ctr[i]; ks[4] ^= key[i]; }
    for (int i = 0; i < 4; i++) x[i] += ks[i];
    for (unsigned r = 0; r < R; r++) {
        const unsigned* rot = ROT_32x4[r % 8];
        if ((r & 1) == 0) {
            x[0] += x[1]; x[1] = rotl32(x[1], rot[0]); x[1] ^= x[0];
            x[2] += x[3]; x[3] = rotl32(x[3], rot[1]); x[3] ^= x[2];
        } else {
            x[0] += x[3]; x[3] = rotl32(x[3], rot[0]); x[3] ^= x[0];
            x[2] += x[1]; x[1] = rotl32(x[1], rot[1]); x[1] ^= x[2];
        }
        if (r % 4 == 3) {
            unsigned s = r / 4 + 1;
            for (int j = 0; j < 4; j++) x[j] += ks[(s + j) % 5];
            x[3] += s;
        }
    }
    memcpy(out, x, sizeof x);
}

void r123_threefry4x32(const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4])
{
    r123_threefry4x32_R(20, ctr, key, out);
}

/* Threefry4x32 as the reference JIT prints it (R123Threefry.cpp:230-283):
 * every round mixes the fixed lane pairs (0,1),(2,3) -- the odd-round
 * (0,3),(2,1) pairing of upstream Random123 is absent.  This is the stream
 * the reference runs on its devices, so it is the parity target. */
void r123_threefry4x32_chai_R(unsigned R, const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4])
{
    uint32_t ks[5], x[4];
    ks[4] = 0x1BD11BDAu;
    for (int i = 0; i < 4; i++) { ks[i] = key[i]; x[i] = ctr[i]; ks[4] ^= key[i]; }
    for (int i = 0; i < 4; i++) x[i] += ks[i];
    for (unsigned r = 0; r < R; r++) {
        const unsigned* rot = ROT_32x4[r % 8];
        x[0] += x[1]; x[1] = rotl32(x[1], rot[0]); x[1] ^= x[0];
        x[2] += x[3]; x[3] = rotl32(x[3], rot[1]); x[3] ^= x[2];
        if (r % 4 == 3) {
            unsigned s = r / 4 + 1;
            for (int j = 0; j < 4; j++) x[j] += ks[(s + j) % 5];
            x[3] += s;
        }
    }
    memcpy(out, x, sizeof x);
}

void r123_threefry4x32_chai(const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4])
{
    r123_threefry4x32_chai_R(20, ctr, key, out);
}

void r123_threefry2x32(const uint32_t ctr[2], const uint32_t key[2], uint32_t out[2])
{
    uint32_t ks[3], x[2];
    ks[2] = 0x1BD11BDAu;
    for (int i = 0; i < 2; i++) { ks[i] = key[i]; x[i] = ctr[i]; ks[2] ^= key[i]; }
    x[0] += ks[0]; x[1] += ks[1];
    for (unsigned r = 0; r < 20; r++) {
        x[0] += x[1]; x[1] = rotl32(x[1], ROT_32x2[r % 8]); x[1] ^= x[0];
        if (r % 4 == 3) {
            unsigned s = r / 4 + 1;
            x[0] += ks[s % 3]; x[1] += ks[(s + 1) % 3];
            x[1] += s;
        }
    }
    out[0] = x[0]; out[1] = x[1];
}

void r123_threefry2x64(const uint64_t ctr[2], const uint64_t key[2], uint64_t out[2])
{
    uint64_t ks[3], x[2];
    ks[2] = 0x1BD11BDAA9FC1A22ull;
    for (int i = 0; i < 2; i++) { ks[i] = key[i]; x[i] = ctr[i]; ks[2] ^= key[i]; }
    x[0] += ks[0]; x[1] += ks[1];
    for (unsigned r = 0; r < 20; r++) {
        x[0] += x[1]; x[1] = rotl64(x[1], ROT_64x2[r % 8]); x[1] ^= x[0];
        if (r % 4 == 3) {
            unsigned s = r / 4 + 1;
            x[0] += ks[s % 3]; x[1] += ks[(s + 1) % 3];
            x[1] += s;
        }
    }
    out[0] = x[0]; out[1] = x[1];
}

/* ------------------------------------------------------------- chai fill */

/* One generator call for vector index `tid` and counter word `idx`:
 * fills up to 4 raw 32-bit lanes (x32) or 2 raw 64-bit lanes (x64). */
static void gen32(int variant, int vec_len, int layout, uint32_t tid, uint32_t idx, uint32_t lanes[4])
{
    uint32_t a = layout ? idx : tid;   /* key word 0 */
    uint32_t b = layout ? tid : idx;   /* counter word 0 */
    if (vec_len == 4) {
        uint32_t ctr[4] = {b, 0xf00dcafeu, 0xdeadbeefu, 0xbeeff00du};
        if (variant == 1231) {
            uint32_t key[4] = {a, 0xdecafbadu, 0xfacebeadu, 0x12345678u};
            r123_threefry4x32_chai(ctr, key, lanes);
        } else {
            uint32_t key[2] = {a, 0xdecafbadu};
            r123_philox4x32(ctr, key, lanes);
        }
    } else {
        uint32_t ctr[2] = {b, 0xf00dcafeu};
        if (variant == 1231) {
            uint32_t key[2] = {a, 0xdecafbadu};
            r123_threefry2x32(ctr, key, lanes);
        } else {
            uint32_t key[1] = {a};
            /* R123Philox.cpp:369-373: the 2x32 key type has one word and the
             * printed initialiser {tid, 0xdecafbad} keeps only tid */
            r123_philox2x32(ctr, key, lanes);
        }
    }
}

static void gen64(int variant, int layout, uint64_t tid, uint64_t idx, uint64_t lanes[2])
{
    uint64_t a = layout ? idx : tid;
    uint64_t b = layout ? tid : idx;
    uint64_t ctr[2] = {b, 0xf00dcafeull};
    if (variant == 1231) {
        uint64_t key[2] = {a, 0xdecafbadull};
        r123_threefry2x64(ctr, key, lanes);
    } else {
        uint64_t key[1] = {a};
        r123_philox2x64(ctr, key, lanes);
    }
}

void chai_rng_fill(int variant, int prec, int vec_len, int dist, int layout,
                   uint64_t seed, uint64_t first_vec, size_t n_elems,
                   int has_limits, double min_limit, double max_limit,
                   double pi, void* out)
{
    const size_t vl = (size_t)vec_len;
    if (prec == 8) {
        double* o = (double*)out;
        const size_t glanes = vl;   /* f64: 2-lane generator, vec_len 1 keeps lane 0 */
        for (size_t e = 0; e < n_elems; e += glanes) {
            const uint64_t tid = first_vec + e / glanes;
            uint64_t raw[2];
            gen64(variant, layout, tid, seed, raw);
            double u[2];
            for (int j = 0; j < 2; j++)
                u[j] = (double)(int64_t)raw[j] * 5.421010862427522170037E-20 + 0.5;
            double v[2];
            if (dist == 1) {
                double r = sqrt(-2.0 * log(u[0]));
                v[0] = r * sin(2.0 * pi * u[1]);
                v[1] = r * cos(2.0 * pi * u[1]);
            } else {
                v[0] = u[0]; v[1] = u[1];
                if (has_limits) {
                    for (int j = 0; j < 2; j++)
                        v[j] = v[j] * (max_limit - min_limit) + (min_limit != 0.0 ? min_limit : 0.0);
                }
            }
            for (size_t j = 0; j < glanes && e + j < n_elems; j++) o[e + j] = v[j];
        }
        return;
    }
    const size_t glanes = vl;   /* lanes consumed per generator call */
    for (size_t e = 0; e < n_elems; e += glanes) {
        const uint64_t tid = first_vec + e / glanes;
        uint32_t raw[4];
        gen32(variant, vec_len, layout, (uint32_t)tid, (uint32_t)seed, raw);
        if (prec == 0 || prec == 1) {
            uint32_t* o = (uint32_t*)out;
            for (size_t j = 0; j < glanes && e + j < n_elems; j++) o[e + j] = raw[j];
            continue;
        }
        float* o = (float*)out;
        float u[4];
        const int nraw = vec_len == 4 ? 4 : 2;
        for (int j = 0; j < nraw; j++) {
            /* convert_float(int) rounds to nearest even; scaling by 2^-32 is
             * exact, so mul+add and a fused multiply-add agree */
            float f = (float)(int32_t)raw[j];
            u[j] = f * 2.3283064365386963e-10f + 0.5f;
        }
        float v[4];
        if (dist == 1) {
            for (int p = 0; p < nraw; p += 2) {
                double r = sqrt(-2.0 * log((double)u[p]));
                double th = 2.0 * pi * (double)u[p + 1];
                v[p] = (float)(r * sin(th));
                v[p + 1] = (float)(r * cos(th));
            }
        } else {
            for (int j = 0; j < nraw; j++) {
                v[j] = u[j];
                if (has_limits) {
                    /* EnqueueAST.cpp:532-543: u * (max-min) [+ min] in float */
                    const float len = (float)(max_limit - min_limit);
                    float t = v[j] * len;
                    if (min_limit != 0.0) t = t + (float)min_limit;
                    v[j] = t;
                }
            }
        }
        for (size_t j = 0; j < glanes && e + j < n_elems; j++) o[e + j] = v[j];
    }
}
