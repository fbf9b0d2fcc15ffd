/* CPU restatement of chai's Random123 generators (the oracle for RNG parity).
 *
 * Test infrastructure only: tests, the smoke check and the bench's CPU
 * baseline call this; the product never links it.
 *
 * Follows the OpenCL that the reference's JIT prints:
 *   Philox bijections     Random123/R123Philox.cpp:34-286  (mulhilo, bumpkey,
 *                         round, _R with 10 rounds)
 *   Threefry bijections   Random123/R123Threefry.cpp:40-295 (rotation tables,
 *                         key-schedule parity 0x1BD11BDA, 20 rounds)
 *   key / counter layout  R123Philox.cpp:369-381, R123Threefry.cpp:375-387
 *   uniform conversion    R123Philox.cpp:405-427 (int * 2^-32 + 0.5, 64-bit:
 *                         int64 * 2^-64 + 0.5; constants R123Util.cpp:97-98)
 *   normal (Box-Muller)   R123Philox.cpp:466-515
 *   interval scaling      enqueue/EnqueueAST.cpp:517-545
 *   generator selection   kernel/Function.cpp:388-431 (32-bit precisions use
 *                         the x32 generators, f64 the x64 ones; vector length 4
 *                         uses the 4-lane generator, 1 and 2 the 2-lane one)
 *   seed bump             api/RngFun.cpp:15-31 (seed += W*H*slots per call)
 */
#ifndef CHAI_ORACLE_R123_H
#define CHAI_ORACLE_R123_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* raw bijections, 10 (Philox) / 20 (Threefry) rounds */
void r123_philox2x32(const uint32_t ctr[2], const uint32_t key[1], uint32_t out[2]);
void r123_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void r123_philox2x64(const uint64_t ctr[2], const uint64_t key[1], uint64_t out[2]);
void r123_threefry2x32(const uint32_t ctr[2], const uint32_t key[2], uint32_t out[2]);
void r123_threefry4x32(const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4]);
void r123_threefry2x64(const uint64_t ctr[2], const uint64_t key[2], uint64_t out[2]);
/* round-count variants used to compare against the upstream _R functions */
void r123_philox4x32_R(unsigned R, const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void r123_threefry4x32_R(unsigned R, const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4]);
/* the reference JIT's printed Threefry4x32 (fixed lane pairing, see r123.c) */
void r123_threefry4x32_chai(const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4]);
void r123_threefry4x32_chai_R(unsigned R, const uint32_t ctr[4], const uint32_t key[4], uint32_t out[4]);

/* Chai array fill.
 *   variant  1230 Philox, 1231 Threefry (api/chai.h:412-417)
 *   prec     0 u32, 1 i32, 4 f32, 8 f64  (misc/PrecType codes)
 *   vec_len  1, 2 or 4: the JIT's vector length for the statement
 *   dist     0 uniform, 1 normal
 *   layout   0 chai (key word 0 = vector index, counter word 0 = seed),
 *            1 counter (key word 0 = seed, counter word 0 = vector index)
 *   pi       the constant used inside Box-Muller (the reference JIT prints
 *            M_PI with 6 significant digits: 3.14159)
 *   limits   has_limits != 0: u * (max - min) + min, as printed by the JIT
 * Element e (row-major over slots*H*W, rows of W elements, W % vec_len == 0)
 * takes lane e % vec_len of the generator called with vector index
 * first_vec + e / vec_len. */
void chai_rng_fill(int variant, int prec, int vec_len, int dist, int layout,
                   uint64_t seed, uint64_t first_vec, size_t n_elems,
                   int has_limits, double min_limit, double max_limit,
                   double pi, void* out);

#ifdef __cplusplus
}
#endif

#endif
