/*
 * ff_oracle.h -- CPU restatement of the reference hot path, used ONLY as a checker.
 *
 * This is test infrastructure: the tests, the smoke check and bench.py's CPU-baseline leg
 * may call it; the product (ff-gpu_b200/) never links or runs it.
 *
 * It restates, from the reference program reference/segmentedSieve.C (ff_seg):
 *   - the leg geometry and the two header lines           (segmentedSieve.C:136-182, 875-879)
 *   - the odd-only bitmap and its segment fill             (segmentedSieve.C:184-222, 255-270)
 *   - IsPrime + deterministic Miller-Rabin                 (segmentedSieve.C:283-296, 310-387)
 *   - FreudenthalTools / Sammy2Loopy per-sum search        (segmentedSieve.C:408-639)
 *   - the RunIt filter and the solution line format        (segmentedSieve.C:645-677, 800-823)
 *   - GenerateThreads' 62-way partition and merge order    (segmentedSieve.C:706-792, 905-912)
 * and, from ff-gpu, the slab-relative layout of SieveSlabRun (source/sieve_slab_kernel.h:40-107).
 *
 * Parity is pinned by tests/test_oracle.py against the reference goldens
 * (goldens/out_ff_seg_*.txt via their SHA-256 and counts) and against outputs of the
 * reference binary built from its own source (oracle/_ref/ff_seg), committed as fixtures.
 */
#ifndef FF_ORACLE_H
#define FF_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Work counters of the instrumented search (summed over the sums evaluated). */
typedef struct {
    uint64_t sums;          /* odd sums evaluated (after the RunIt loop, before the filter) */
    uint64_t map_probes;    /* IsPrime answered from the bitmap                               */
    uint64_t mr_calls;      /* IsPrime answered by Miller-Rabin (n above the map)             */
    uint64_t mr_mulmods;    /* modular multiplications inside those Miller-Rabin calls        */
    uint64_t splits;        /* (evenTerm, oddTerm) decompositions handed to DoesPeterKnow /   */
                            /* AllButOne... (the quick checks included)                      */
    uint64_t abop_calls;    /* AllButOneProductOfTermPairs... invocations                      */
    uint64_t trial_steps;   /* iterations of the trial-division loop inside those calls       */
    uint64_t divisors;      /* divisor pairs tested inside those calls                        */
    uint64_t errors;        /* inputs outside the exact domain (n >= 2^48 for MR, overflow)   */
} ffo_counters;

typedef struct ffo_ctx ffo_ctx;

/* Geometry of one ff_seg invocation (segmentedSieve.C:844-879 and Prime::Prime :136-182). */
typedef struct {
    uint32_t sum_start;          /* after |1 and the >=5 clamp                          */
    uint32_t sum_limit;          /* after the >= sumStart clamp                         */
    uint32_t max_generated_prime;
    uint64_t product_limit;
    uint64_t prime_limit;
    uint64_t num_primes_requested;
    uint64_t max_prime_map_value;   /* mpv after the estimate/renormalisation branches  */
    uint64_t prime_map_bytes;       /* bytes the reference allocates for the map        */
    uint64_t sqrt_limit;
    uint64_t pmap_sum_limit;        /* isqrt64((mpv-2)<<2)<<1 (segmentedSieve.C:905)    */
    int      renormalised;          /* the PRIMEMEM branch was taken                    */
    int      too_big;               /* the reference would exit(-1) here                */
} ffo_geometry;

uint64_t ffo_isqrt64(uint64_t n);

/* argc-style argument handling of main (segmentedSieve.C:844-855): nargs = number of
 * positional arguments given (0, 1 or 2); a1/a2 are their atoi() values. */
void ffo_parse_args(int nargs, int32_t a1, int32_t a2, uint32_t* sum_start, uint32_t* sum_limit);

/* Fills g and writes the header text (2 or 3/4 lines, each ending in '\n') into buf.
 * Returns the number of bytes written (excluding the NUL), or -1 if cap is too small. */
int ffo_geometry_headers(uint32_t sum_start, uint32_t sum_limit, ffo_geometry* g,
                         char* buf, size_t cap);

/* GenerateThreads' partition of [sum_start, sum_limit] for `threads` twins, followed by
 * the two-call split of main. Writes (first,last) sub-ranges in EMISSION order (fronts in
 * launch order, then backs in reverse launch order; the second call's ranges after the
 * first call's). Returns the number of ranges, or -1 if cap is too small / the range is
 * outside what the reference can run. */
int ffo_schedule(uint32_t sum_start, uint32_t sum_limit, uint64_t max_prime_map_value,
                 uint32_t threads, uint32_t* firsts, uint32_t* lasts, int cap);

/* Prime::SegmentFill with GLOBAL indexing: clears, for each p of the list, the bit of
 * every odd multiple i >= p*p of p with segLo <= i < segHi (byte i>>4, bit 0x80>>(i>>1&7)). */
void ffo_segment_fill(uint64_t seg_lo, uint64_t seg_hi, const uint32_t* primes, uint32_t n,
                      uint8_t* map);

/* The slab contract of SieveSlabRun: out has (seg_hi+15)>>4 bytes; it is set to 0xff
 * (byte 0 = 0x7f when seg_lo == 0) and the marks of [seg_lo, seg_hi) are written with
 * seg_lo-RELATIVE indexing (value i -> bit position (i-seg_lo)>>1). */
void ffo_slab_relative(uint64_t seg_lo, uint64_t seg_hi, const uint32_t* primes, uint32_t n,
                       uint8_t* out);

/* Odd primes <= limit in ascending order (2 excluded). Returns the count written (at most
 * cap), or the total count when out == NULL. */
uint64_t ffo_odd_primes(uint64_t limit, uint32_t* out, uint64_t cap);

/* The reference prime map for max_prime_map_value: (mpv+1+15)>>4 bytes, all values up to
 * mpv sieved, value 1 cleared. Multithreaded over byte-aligned chunks. */
int ffo_build_map(uint64_t max_prime_map_value, uint8_t* map, int nthreads);

/* Deterministic Miller-Rabin with the reference's witness list and thresholds. */
int ffo_miller_rabin(uint64_t n);

/* A search context: a bitmap covering values <= map_bound (0 => the reference's full
 * map for max_sum's geometry) and the trial-division prime list for sums <= max_sum. */
ffo_ctx* ffo_create(uint32_t max_sum, uint64_t map_bound, int nthreads);
void     ffo_destroy(ffo_ctx* c);
uint64_t ffo_map_bound(const ffo_ctx* c);
const uint8_t* ffo_map(const ffo_ctx* c);
int      ffo_is_prime(const ffo_ctx* c, uint64_t n);

/* One odd sum through the RunIt filter and DoesSammyKnow. Returns 1 and the ordered terms
 * when the sum produces a solution line, else 0. */
int ffo_eval_sum(const ffo_ctx* c, uint32_t sum, uint32_t* low, uint32_t* high,
                 ffo_counters* k);

/* All odd sums s in [lo, hi] (lo odd): out[(s-lo)/2] = (uint64)low<<32 | high, or 0.
 * Multithreaded; counters (if not NULL) receive the totals. */
int ffo_eval_range(const ffo_ctx* c, uint32_t lo, uint32_t hi, uint64_t* out, int nthreads,
                   ffo_counters* k);

/* One solution line, with the count field, terminated by '\n'. Returns its length. */
int ffo_format_line(const ffo_ctx* c, uint32_t count, uint32_t sum, uint32_t low,
                    uint32_t high, char* buf, size_t cap);

/* The whole ff_seg stdout for the given argument list (see ffo_parse_args), with the two
 * timing lines normalised to "N" (the reference goldens' form). map_bound as in
 * ffo_create (0 => full reference map). Returns a malloc'd NUL-terminated buffer
 * (free with ffo_free) and its length in *len; NULL on error. */
char* ffo_run(int nargs, int32_t a1, int32_t a2, uint64_t map_bound, int nthreads,
              size_t* len, ffo_counters* k);
void  ffo_free(void* p);

/* The same text from per-sum records already evaluated (rec[(s - rec_lo)/2] for the odd sums
 * rec_lo .. rec_lo + 2*(nrec-1), which must cover the schedule of the argument list), with c
 * answering the prime tags of the terms. Lets many argument lists share one evaluation of
 * the union of their sums. NULL when the records do not cover the schedule. */
char* ffo_emit(const ffo_ctx* c, int nargs, int32_t a1, int32_t a2, const uint64_t* rec,
               uint32_t rec_lo, uint64_t nrec, size_t* len);

#ifdef __cplusplus
}
#endif

#endif
