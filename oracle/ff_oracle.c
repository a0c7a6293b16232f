/*
 * ff_oracle.c -- CPU restatement of the reference hot path (checker only; see ff_oracle.h).
 *
 * Every function names the reference lines it restates. The restatement keeps the
 * reference's integer types, its loop orders and its double-precision expressions
 * (compiled with -ffp-contract=off) wherever they decide an output byte; elsewhere it is
 * free to differ (e.g. the bitmap is built by any exact sieve, since the reference's
 * map is the exact odd-prime bitmap up to maxPrimeMapValue).
 */
#define _GNU_SOURCE
#include "ff_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define FFO_PRIMEMEM (85ull * 1073741824ull)  /* segmentedSieve.C:9-11 (PRIMEMEM)  */
#define FFO_THREADS  31u                      /* segmentedSieve.C:12-14 (THREADS)   */
#define FFO_MAX_FACTOR_LIST 8192               /* > 2*g*(g-1) for every product < 2^48 */

/* ------------------------------------------------------------------------------------ */
/* small helpers                                                                         */
/* ------------------------------------------------------------------------------------ */

/* floor(sqrt(n)) for every 64-bit n (segmentedSieve.C:37-52 computes the same value). */
uint64_t ffo_isqrt64(uint64_t n)
{
    if (n < 2) return n;
    uint64_t r = (uint64_t)sqrt((double)n);
    /* correct the double estimate; (r+1)^2 cannot overflow while r < 2^32-1 */
    while (r > 0 && (r > 0xFFFFFFFFull || r * r > n)) --r;
    while (r < 0xFFFFFFFFull && (r + 1) * (r + 1) <= n) ++r;
    return r;
}

static inline int map_bit(const uint8_t* map, uint64_t v)
{
    return (map[v >> 4] >> (7 - ((v >> 1) & 7))) & 1;
}

/* ------------------------------------------------------------------------------------ */
/* argument handling and geometry (segmentedSieve.C:136-182, 844-879, 905)               */
/* ------------------------------------------------------------------------------------ */

void ffo_parse_args(int nargs, int32_t a1, int32_t a2, uint32_t* sum_start, uint32_t* sum_limit)
{
    uint32_t s, l;
    if (nargs >= 2) {                 /* sumStart=atoi(argv[1])|1; sumLimit=atoi(argv[2]) */
        s = (uint32_t)a1 | 1u;
        l = (uint32_t)a2;
    } else {                          /* sumStart=5; sumLimit=argc>1 ? atoi(argv[1]) : 2627 */
        s = 5;
        l = nargs == 1 ? (uint32_t)a1 : 2627u;
    }
    if (s < 5) s = 5;
    if (s > l) l = s;
    *sum_start = s;
    *sum_limit = l;
}

static int append(char* buf, size_t cap, size_t* pos, const char* fmt, ...)
    __attribute__((format(printf, 4, 5)));

#include <stdarg.h>
static int append(char* buf, size_t cap, size_t* pos, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int n = vsnprintf(buf ? buf + *pos : NULL, buf ? cap - *pos : 0, fmt, ap);
    va_end(ap);
    if (n < 0 || (buf && (size_t)n >= cap - *pos)) return -1;
    *pos += (size_t)n;
    return 0;
}

/* The prime-count estimate and the map sizing of Prime::Prime (segmentedSieve.C:136-182)
 * with the arguments main passes (segmentedSieve.C:875-879). */
int ffo_geometry_headers(uint32_t sum_start, uint32_t sum_limit, ffo_geometry* g,
                         char* buf, size_t cap)
{
    memset(g, 0, sizeof *g);
    g->sum_start = sum_start;
    g->sum_limit = sum_limit;
    uint32_t mgp = (sum_limit + 1u) >> 1;
    uint64_t product_limit = (uint64_t)mgp * mgp;
    uint64_t prime_limit = (product_limit >> 2) + 2;
    double xlogx = (double)mgp / log((double)mgp);
    uint32_t n_primes = (uint32_t)(xlogx + 1.2762 * xlogx / log((double)mgp));
    g->max_generated_prime = mgp;
    g->product_limit = product_limit;
    g->prime_limit = prime_limit;

    uint64_t n_req = n_primes > 1 ? n_primes : 1;
    uint64_t map_size = ((prime_limit > 1 ? prime_limit : 2) + 15) >> 4;
    uint64_t mpv = (map_size << 4) - 1;
    uint64_t est = (uint64_t)((double)n_req * (log((double)n_req) + log(log((double)n_req))));
    if (mpv < est) mpv = est;
    map_size = (mpv + 15) >> 4;
    uint64_t req_size = 4u * n_req;
    uint64_t total = req_size + map_size;
    size_t pos = 0;
    if (append(buf, cap, &pos, "maxPrimeMapValue %llu numPrimesRequested %llu totalBytes %llu\n",
               (unsigned long long)mpv, (unsigned long long)n_req, (unsigned long long)total))
        return -1;
    if (total > FFO_PRIMEMEM) {
        if (16 * FFO_PRIMEMEM > 3 * est) {
            uint64_t new_n = 2 * n_req / 5, new_size = 4u * new_n;
            est = (uint64_t)((double)new_n * (log((double)new_n) + log(log((double)new_n))));
            if (new_size + (est + 1) / 2 > FFO_PRIMEMEM) {
                n_req = ((req_size * FFO_PRIMEMEM + total - 1) / total + 4 - 1) & ~(uint64_t)3;
                req_size = 4u * n_req;
                if (append(buf, cap, &pos,
                           "You probably should consider how badly this run is going to "
                           "perform, just sayin'.\n"))
                    return -1;
            } else {
                n_req = new_n;
                req_size = new_size;
            }
            map_size = FFO_PRIMEMEM - req_size;
            total = req_size + map_size;
            mpv = (map_size << 4) - 1;
            if (append(buf, cap, &pos,
                       "numPrimesRequested %llu maxPrimeMapValue %llu totalBytes %llu\n",
                       (unsigned long long)n_req, (unsigned long long)mpv,
                       (unsigned long long)total))
                return -1;
            g->renormalised = 1;
        } else {
            if (append(buf, cap, &pos,
                       "\nThe input parameters would indicate that more memory is required. "
                       "Please adjust input parameters or Prime::maxPrimeAlloc.\n\n"))
                return -1;
            g->too_big = 1;
            return (int)pos;
        }
    }
    uint64_t sqrt_limit = ffo_isqrt64(mpv);
    if (append(buf, cap, &pos, "maxPrimeMapValue %llu numPrimesRequested %llu sqrtLimit %llu\n",
               (unsigned long long)mpv, (unsigned long long)n_req,
               (unsigned long long)sqrt_limit))
        return -1;
    g->num_primes_requested = n_req;
    g->max_prime_map_value = mpv;
    g->prime_map_bytes = map_size;
    g->sqrt_limit = sqrt_limit;
    g->pmap_sum_limit = ffo_isqrt64((mpv - 2) << 2) << 1;
    return (int)pos;
}

/* ------------------------------------------------------------------------------------ */
/* GenerateThreads partition (segmentedSieve.C:706-792) and main's split (:905-912)       */
/* ------------------------------------------------------------------------------------ */

typedef struct { uint32_t first, last; } range_t;

/* One GenerateThreads call: appends front ranges to fr[] (launch order) and back ranges
 * to bk[] (launch order; emitted in reverse). */
static int generate_threads(uint32_t sum_start, uint32_t sum_limit, uint32_t threads,
                            range_t* fr, int* nf, range_t* bk, int* nb)
{
    uint32_t num_sum = sum_limit - sum_start + 1u;
    if (num_sum > 0x7FFFFFFFu) return -1;     /* only reachable through uint32 wrap */
    double delta = (double)num_sum / (2 * threads);
    uint32_t s1 = 0, s2 = num_sum, s1_prev = 0, s2_prev = num_sum;
    uint32_t l1 = 0, l2 = 0;
    int f1 = 1, f2 = 1;
    *nf = *nb = 0;
    for (uint32_t t = 0; t < threads; ++t) {
        s1 = (uint32_t)(t * delta + .5);
        if (s1 > s1_prev) { s1_prev = s1; f1 = 1; }
        uint32_t t2 = 2 * threads - t - 1;
        s2 = (uint32_t)(t2 * delta + .5);
        if (s2 < s2_prev) { s2_prev = s2; f2 = 1; }
        if (f1 && f2) {
            f1 = f2 = 0;
            l1 = (uint32_t)((t + 1) * delta - .5);
            if (l1 < s1) l1 = s1;
            int second = s1 < s2;
            if (second) {
                l2 = (uint32_t)((t2 + 1) * delta - .5);
                if (l2 < s2) l2 = s2;
            }
            fr[*nf].first = s1 + sum_start;
            fr[*nf].last = l1 + sum_start;
            ++*nf;
            if (second) {
                bk[*nb].first = s2 + sum_start;
                bk[*nb].last = l2 + sum_start;
                ++*nb;
            }
        }
    }
    return 0;
}

int ffo_schedule(uint32_t sum_start, uint32_t sum_limit, uint64_t mpv, uint32_t threads,
                 uint32_t* firsts, uint32_t* lasts, int cap)
{
    if (threads == 0 || threads > 4096) return -1;
    uint64_t pmap = ffo_isqrt64((mpv - 2) << 2) << 1;
    uint32_t calls[2][2];
    int ncalls;
    if (sum_limit <= pmap) {
        calls[0][0] = sum_start; calls[0][1] = sum_limit; ncalls = 1;
    } else {
        calls[0][0] = sum_start; calls[0][1] = (uint32_t)pmap;
        calls[1][0] = (uint32_t)((pmap + 1) | 1); calls[1][1] = sum_limit;
        ncalls = 2;
    }
    range_t* fr = malloc(sizeof(range_t) * threads);
    range_t* bk = malloc(sizeof(range_t) * threads);
    int n = 0;
    for (int c = 0; c < ncalls; ++c) {
        int nf, nb;
        if (generate_threads(calls[c][0], calls[c][1], threads, fr, &nf, bk, &nb)) { n = -1; break; }
        if (n + nf + nb > cap) { n = -1; break; }
        for (int i = 0; i < nf; ++i) { firsts[n] = fr[i].first; lasts[n] = fr[i].last; ++n; }
        for (int i = nb - 1; i >= 0; --i) { firsts[n] = bk[i].first; lasts[n] = bk[i].last; ++n; }
    }
    free(fr);
    free(bk);
    return n;
}

/* ------------------------------------------------------------------------------------ */
/* sieve (segmentedSieve.C:184-222, 255-270; source/sieve_slab_kernel.h:40-107)          */
/* ------------------------------------------------------------------------------------ */

/* Prime::SegmentFill: odd multiples i >= p*p of each listed p inside [seg_lo, seg_hi).
 * The reference walks 2^19-value sub-blocks and stops at the first p with p*p >= bHi;
 * for an ascending list that stop removes no mark (every mark of p is >= p*p), so the
 * restatement marks each listed p over the whole segment. */
void ffo_segment_fill(uint64_t seg_lo, uint64_t seg_hi, const uint32_t* primes, uint32_t n,
                      uint8_t* map)
{
    for (uint32_t k = 0; k < n; ++k) {
        uint64_t p = primes[k];
        if (p == 0) continue;
        uint64_t pp = p * p;
        if (pp >= seg_hi) continue;
        uint64_t first = (seg_lo + p - 1) / p * p;
        if (first < pp) first = pp;
        if (!(first & 1)) first += p;
        for (uint64_t i = first; i < seg_hi; i += p << 1)
            map[i >> 4] &= (uint8_t)~(0x80u >> ((i >> 1) & 7));
    }
}

/* SieveSlabRun's output contract (source/sieve_slab_kernel.cpp:80-105 and the kernel's
 * running offset, source/sieve_slab_kernel.h:95-105): value i -> relative offset i-seg_lo,
 * byte offset>>4, bit 0x80>>(offset>>1&7). */
void ffo_slab_relative(uint64_t seg_lo, uint64_t seg_hi, const uint32_t* primes, uint32_t n,
                       uint8_t* out)
{
    uint64_t bytes = (seg_hi + 15) >> 4;
    memset(out, 0xff, bytes);
    if (seg_lo == 0) out[0] ^= 0x80;
    for (uint32_t k = 0; k < n; ++k) {
        uint64_t p = primes[k];
        if (p == 0) continue;
        uint64_t pp = p * p;
        if (pp >= seg_hi) continue;
        uint64_t first = (seg_lo + p - 1) / p * p;
        if (first < pp) first = pp;
        if (!(first & 1)) first += p;
        for (uint64_t i = first; i < seg_hi; i += p << 1) {
            uint64_t off = i - seg_lo;
            out[off >> 4] &= (uint8_t)~(0x80u >> ((off >> 1) & 7));
        }
    }
}

uint64_t ffo_odd_primes(uint64_t limit, uint32_t* out, uint64_t cap)
{
    if (limit < 3) return 0;
    uint64_t nodd = (limit - 1) / 2;          /* odd numbers 3..limit: index j -> 2j+3 */
    uint8_t* comp = calloc(nodd + 1, 1);
    for (uint64_t j = 0; j < nodd; ++j) {
        if (comp[j]) continue;
        uint64_t p = 2 * j + 3;
        if (p * p > limit) break;
        for (uint64_t m = p * p; m <= limit; m += 2 * p) comp[(m - 3) / 2] = 1;
    }
    uint64_t cnt = 0;
    for (uint64_t j = 0; j < nodd; ++j) {
        if (comp[j]) continue;
        if (out && cnt < cap) out[cnt] = (uint32_t)(2 * j + 3);
        ++cnt;
    }
    free(comp);
    return out && cnt > cap ? cap : cnt;
}

typedef struct {
    uint64_t lo, hi;
    const uint32_t* primes;
    uint32_t n;
    uint8_t* map;
} fill_job;

static void* fill_worker(void* arg)
{
    fill_job* j = arg;
    ffo_segment_fill(j->lo, j->hi, j->primes, j->n, j->map);
    return NULL;
}

/* Prime::Prime's map (segmentedSieve.C:183-219): memset 0xff, value 1 cleared, odd
 * primes <= isqrt(mpv) marked over byte-aligned chunks in parallel. */
int ffo_build_map(uint64_t mpv, uint8_t* map, int nthreads)
{
    uint64_t bytes = (mpv + 1 + 15) >> 4;
    memset(map, 0xff, bytes);
    map[0] ^= 0x80;
    uint64_t sq = ffo_isqrt64(mpv);
    uint64_t np = ffo_odd_primes(sq, NULL, 0);
    uint32_t* pr = malloc(sizeof(uint32_t) * (np ? np : 1));
    ffo_odd_primes(sq, pr, np);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    uint64_t chunk = ((mpv + 1 + (uint64_t)nthreads - 1) / (uint64_t)nthreads + 15) & ~(uint64_t)15;
    pthread_t th[256];
    fill_job jobs[256];
    int started = 0;
    for (int t = 0; t < nthreads; ++t) {
        uint64_t lo = (uint64_t)t * chunk, hi = lo + chunk;
        if (hi > mpv + 1) hi = mpv + 1;
        if (lo >= hi) continue;
        jobs[started] = (fill_job){lo, hi, pr, (uint32_t)np, map};
        pthread_create(&th[started], NULL, fill_worker, &jobs[started]);
        ++started;
    }
    for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
    free(pr);
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* Miller-Rabin (segmentedSieve.C:310-387)                                               */
/* ------------------------------------------------------------------------------------ */

/* The reference's ModularMulL is exact for moduli below 2^48; within that domain this
 * 128-bit product gives the same residues. Callers stay below 2^48 (checked). */
static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t m)
{
    return (uint64_t)((unsigned __int128)a * b % m);
}

static int miller_rabin_counted(uint64_t n, ffo_counters* k)
{
    static const uint64_t bases[7] = {2, 3, 5, 7, 11, 13, 17};
    if (k) {
        ++k->mr_calls;
        if (n >= (1ull << 48)) ++k->errors;
    }
    uint32_t s = (uint32_t)__builtin_ctzll(n >> 1) + 1;      /* power2      */
    uint64_t d = n >> s;                                      /* nDiv2Odd    */
    uint32_t tests = n < 3215031751ull ? 4 : n < 2152302898747ull ? 5
                   : n < 3474749660383ull ? 6 : 7;
    uint64_t mm = 0;
    for (uint32_t i = 0; i < tests; ++i) {
        /* ModularPower(p, nDiv2Odd, n): right-to-left square-and-multiply */
        uint64_t x = 1, b = bases[i], e = d;
        while (e) {
            if (e & 1) { x = mulmod(x, b, n); ++mm; }
            e >>= 1;
            b = mulmod(b, b, n); ++mm;
        }
        if (x != 1 && x != n - 1) {
            for (uint32_t r = 1; r < s; ++r) {
                x = mulmod(x, x, n); ++mm;
                if (x == 1) { if (k) k->mr_mulmods += mm; return 0; }
                if (x == n - 1) break;
            }
            if (x != n - 1) { if (k) k->mr_mulmods += mm; return 0; }
        }
    }
    if (k) k->mr_mulmods += mm;
    return 1;
}

int ffo_miller_rabin(uint64_t n) { return miller_rabin_counted(n, NULL); }

/* ------------------------------------------------------------------------------------ */
/* search context                                                                         */
/* ------------------------------------------------------------------------------------ */

struct ffo_ctx {
    uint8_t* map;
    uint64_t bound;        /* values <= bound are answered by the bitmap */
    uint32_t* primes;      /* primes[0]=2, primes[1]=3, ... (Prime::operator[]) */
    uint32_t nprimes;
    uint32_t max_sum;
};

/* Prime::IsPrime (segmentedSieve.C:283-296) */
static inline int is_prime(const ffo_ctx* c, uint64_t n, ffo_counters* k)
{
    if (n == 2) return 1;
    if (!(n & 1)) return 0;
    if (n > c->bound) return miller_rabin_counted(n, k);
    if (k) ++k->map_probes;
    return map_bit(c->map, n);
}

int ffo_is_prime(const ffo_ctx* c, uint64_t n) { return is_prime(c, n, NULL); }
uint64_t ffo_map_bound(const ffo_ctx* c) { return c->bound; }
const uint8_t* ffo_map(const ffo_ctx* c) { return c->map; }

ffo_ctx* ffo_create(uint32_t max_sum, uint64_t map_bound, int nthreads)
{
    ffo_ctx* c = calloc(1, sizeof *c);
    if (!c) return NULL;
    if (map_bound == 0) {
        ffo_geometry g;
        char hb[1024];
        if (ffo_geometry_headers(5, max_sum < 5 ? 5 : max_sum, &g, hb, sizeof hb) < 0 || g.too_big) {
            free(c);
            return NULL;
        }
        map_bound = g.max_prime_map_value;
    }
    if (map_bound < 15) map_bound = 15;
    uint64_t map_mpv = (((map_bound + 1 + 15) >> 4) << 4) - 1;   /* whole bytes */
    c->map = malloc((map_mpv + 1 + 15) >> 4);
    if (!c->map) { free(c); return NULL; }
    ffo_build_map(map_mpv, c->map, nthreads);
    c->bound = map_bound;
    c->max_sum = max_sum;
    /* trial-division primes: every prime up to max_sum/2 plus a margin (factorLimit of a
     * product a*b with a+b=sum is at most sum/2) */
    uint64_t plim = (uint64_t)max_sum / 2 + 4096;
    uint64_t np = ffo_odd_primes(plim, NULL, 0);
    c->primes = malloc(sizeof(uint32_t) * (np + 1));
    c->primes[0] = 2;
    ffo_odd_primes(plim, c->primes + 1, np);
    c->nprimes = (uint32_t)(np + 1);
    return c;
}

void ffo_destroy(ffo_ctx* c)
{
    if (!c) return;
    free(c->map);
    free(c->primes);
    free(c);
}

/* Prime::operator[] (segmentedSieve.C:272-281): the index-th prime. */
static inline uint64_t nth_prime(const ffo_ctx* c, uint32_t index, ffo_counters* k)
{
    if (index < c->nprimes) return c->primes[index];
    uint32_t n = c->nprimes - 1;
    uint64_t p = (uint64_t)c->primes[n] + 2;
    for (;; p += 2) {
        if (is_prime(c, p, k) && ++n >= index) return p;
    }
}

/* ------------------------------------------------------------------------------------ */
/* FreudenthalTools (segmentedSieve.C:408-477)                                            */
/* ------------------------------------------------------------------------------------ */

/* ProductOfTermPairsHasSingleFactorPair (segmentedSieve.C:419-422) */
static inline int ptphsfp(const ffo_ctx* c, uint64_t i, ffo_counters* k)
{
    if (!(i & 1)) return 1;
    return is_prime(c, i - 2, k);
}

/* AllButOneProductOfTermPairsOfSumOfFactorPairsHasSingleFactorPair (segmentedSieve.C:
 * 424-477): walks the divisors d <= isqrt(oddProduct<<power2) that the reference's
 * trial-division loop generates (including its partially-sorted skip at :451) and counts
 * those whose pair sum d + product/d is NOT "prime + 2"; true iff exactly one. */
static int abop(const ffo_ctx* c, uint32_t power2, uint64_t odd_product, ffo_counters* k)
{
    uint64_t factors[FFO_MAX_FACTOR_LIST];
    uint32_t prime_index = 1, nf = 0, npend = 0, nmfp = 0;
    uint64_t prime_factor = 3;
    uint64_t product = odd_product << power2;
    uint64_t test_product = odd_product;
    uint64_t temp = test_product / 3;
    uint64_t test_factor = 3;
    uint64_t factor_limit = ffo_isqrt64(product);
    if (k) ++k->abop_calls;
    factors[0] = (uint64_t)(1u << power2);
    if (factors[0] <= factor_limit) {
        if (k) ++k->divisors;
        nmfp += !ptphsfp(c, factors[nf++] + odd_product, k);
    }
    for (;;) {
        if (k) ++k->trial_steps;
        if (temp * prime_factor == test_product) {
            if (test_factor <= factor_limit) {
                if (k) ++k->divisors;
                if ((nmfp += !ptphsfp(c, test_factor + product / test_factor, k)) > 1) return 0;
                if (nf + npend >= FFO_MAX_FACTOR_LIST) { if (k) ++k->errors; return 0; }
                factors[nf + npend++] = test_factor;
                for (uint32_t f = 0; f < nf; ++f) {
                    uint64_t m = factors[f] * test_factor;
                    if (m <= factor_limit) {
                        if (k) ++k->divisors;
                        if ((nmfp += !ptphsfp(c, m + product / m, k)) > 1) return 0;
                        if (nf + npend >= FFO_MAX_FACTOR_LIST) { if (k) ++k->errors; return 0; }
                        factors[nf + npend++] = m;
                    } else {
                        /* skip to the end of this ascending run of factors[] */
                        for (uint64_t v = factors[f]; f + 1 < nf && v <= factors[f + 1]; ++f) {}
                    }
                }
                if (nmfp > 1) return 0;
            }
            test_product = temp;
            temp /= prime_factor;
            test_factor *= prime_factor;
        } else {
            if (test_product == 1) break;
            if (is_prime(c, test_product, k)) {
                if (test_product > factor_limit) break;
                prime_factor = test_product;
                temp = 1;
            } else {
                prime_factor = nth_prime(c, ++prime_index, k);
                if (prime_factor > factor_limit) break;
                temp = test_product / prime_factor;
            }
            nf += npend;
            npend = 0;
            test_factor = prime_factor;
        }
    }
    return nmfp == 1;
}

/* ------------------------------------------------------------------------------------ */
/* Sammy2Loopy (segmentedSieve.C:483-639) and the RunIt filter (:800-823)                 */
/* ------------------------------------------------------------------------------------ */

typedef struct {
    uint32_t count;        /* numProductsWithOnlyOneMultipleFactorPair */
    uint32_t term_a, term_b;
    int found;
    int32_t ncomp;
    uint32_t comp[64];     /* compositePower2 */
} sammy_t;

static inline void note_first(sammy_t* s, uint32_t a, uint32_t b)
{
    if (!s->found && s->count == 1) { s->term_a = a; s->term_b = b; s->found = 1; }
}

/* DoesPeterKnow (segmentedSieve.C:632-639) */
static int peter_knows(const ffo_ctx* c, uint32_t power2, uint32_t odd_part, uint32_t odd,
                       uint64_t odd_product, ffo_counters* k)
{
    if (k) ++k->splits;
    if (!ptphsfp(c, ((uint64_t)1 << power2) + odd_product, k)) return 0;
    if (odd_part != odd && !ptphsfp(c, odd_part + ((uint64_t)odd << power2), k)) return 0;
    return abop(c, power2, odd_product, k);
}

/* Power2Prime (segmentedSieve.C:547-564) */
static void phase_prime(const ffo_ctx* c, sammy_t* s, uint32_t sum, ffo_counters* k)
{
    s->ncomp = 0;
    for (uint32_t even = 4, p2 = 2; even < sum - 2; even <<= 1, ++p2) {
        uint32_t odd = sum - even;
        if (is_prime(c, odd, k)) {
            if (++s->count > 1) break;
            note_first(s, even, odd);
        } else {
            s->comp[s->ncomp++] = p2;
        }
    }
}

/* Power2Odd (segmentedSieve.C:566-589) */
static void phase_odd(const ffo_ctx* c, sammy_t* s, uint32_t sum, ffo_counters* k)
{
    uint32_t p2;
    for (p2 = 2; (5u << p2) < sum - 2; ++p2) {}
    p2 = (p2 - 2) | 1;
    for (; p2 >= 2; p2 -= 2) {
        uint32_t even;
        for (uint32_t o = 5; (even = o << p2) < sum - 2; o += 2) {
            uint32_t odd = sum - even;
            uint64_t prod = (uint64_t)o * odd;
            if (prod % 3) {
                if ((s->count += peter_knows(c, p2, o, odd, prod, k)) > 1) break;
                note_first(s, even, odd);
            }
        }
    }
}

/* Power2Composite (segmentedSieve.C:591-605) */
static void phase_composite(const ffo_ctx* c, sammy_t* s, uint32_t sum, ffo_counters* k)
{
    for (--s->ncomp; s->ncomp >= 0; --s->ncomp) {
        uint32_t p2 = s->comp[s->ncomp];
        uint32_t even = 1u << p2, odd = sum - even;
        if (k) ++k->splits;
        if ((s->count += abop(c, p2, odd, k)) > 1) break;
        note_first(s, even, odd);
    }
}

/* Power2Even (segmentedSieve.C:607-630) */
static void phase_even(const ffo_ctx* c, sammy_t* s, uint32_t sum, ffo_counters* k)
{
    uint32_t p2;
    for (p2 = 2; (3u << p2) < sum - 2; ++p2) {}
    p2 = (p2 - 1) & ~1u;
    for (; p2 >= 2; p2 -= 2) {
        uint32_t even;
        for (uint32_t o = 3; (even = o << p2) < sum - 2; o += 2) {
            uint32_t odd = sum - even;
            uint64_t prod = (uint64_t)o * odd;
            if (!(prod % 3) || is_prime(c, odd, k)) {
                if ((s->count += peter_knows(c, p2, o, odd, prod, k)) > 1) break;
                note_first(s, even, odd);
            }
        }
    }
}

int ffo_eval_sum(const ffo_ctx* c, uint32_t sum, uint32_t* low, uint32_t* high, ffo_counters* k)
{
    if (k) ++k->sums;
    uint32_t d3 = sum / 3;
    /* Sammy's first statement (segmentedSieve.C:805) */
    if (ptphsfp(c, sum, k)) return 0;
    if (sum == 3 * d3 && !is_prime(c, d3, k)) return 0;
    /* DoesSammyKnow (segmentedSieve.C:529-538) */
    sammy_t s;
    s.count = 0;
    s.found = 0;
    s.term_a = s.term_b = 0;
    phase_prime(c, &s, sum, k);
    if (s.count <= 1) {
        phase_odd(c, &s, sum, k);
        if (s.count <= 1) {
            phase_composite(c, &s, sum, k);
            if (s.count <= 1) phase_even(c, &s, sum, k);
        }
    }
    if (s.count != 1) return 0;
    uint32_t a = s.term_a, b = s.term_b;
    if (a > b) { uint32_t t = a; a = b; b = t; }
    *low = a;
    *high = b;
    return 1;
}

/* ------------------------------------------------------------------------------------ */
/* parallel evaluation of a sum range                                                     */
/* ------------------------------------------------------------------------------------ */

typedef struct {
    const ffo_ctx* c;
    uint32_t lo, hi;
    uint64_t* out;
    atomic_uint_fast64_t next;
    ffo_counters totals;
    pthread_mutex_t mu;
} range_job;

static void* range_worker(void* arg)
{
    range_job* j = arg;
    ffo_counters k;
    memset(&k, 0, sizeof k);
    const uint64_t nsums = ((uint64_t)j->hi - j->lo) / 2 + 1;
    const uint64_t chunk = 16;
    for (;;) {
        uint64_t i0 = atomic_fetch_add(&j->next, chunk);
        if (i0 >= nsums) break;
        uint64_t i1 = i0 + chunk < nsums ? i0 + chunk : nsums;
        for (uint64_t i = i0; i < i1; ++i) {
            uint32_t s = j->lo + (uint32_t)(2 * i), a, b;
            j->out[i] = ffo_eval_sum(j->c, s, &a, &b, &k) ? ((uint64_t)a << 32 | b) : 0;
        }
    }
    pthread_mutex_lock(&j->mu);
    uint64_t* dst = (uint64_t*)&j->totals;
    const uint64_t* src = (const uint64_t*)&k;
    for (size_t f = 0; f < sizeof k / sizeof(uint64_t); ++f) dst[f] += src[f];
    pthread_mutex_unlock(&j->mu);
    return NULL;
}

int ffo_eval_range(const ffo_ctx* c, uint32_t lo, uint32_t hi, uint64_t* out, int nthreads,
                   ffo_counters* k)
{
    if (!(lo & 1) || hi < lo) return -1;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 512) nthreads = 512;
    range_job j;
    j.c = c;
    j.lo = lo;
    j.hi = hi;
    j.out = out;
    atomic_init(&j.next, 0);
    memset(&j.totals, 0, sizeof j.totals);
    pthread_mutex_init(&j.mu, NULL);
    pthread_t th[512];
    for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, range_worker, &j);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    pthread_mutex_destroy(&j.mu);
    if (k) {
        uint64_t* dst = (uint64_t*)k;
        const uint64_t* src = (const uint64_t*)&j.totals;
        for (size_t f = 0; f < sizeof *k / sizeof(uint64_t); ++f) dst[f] += src[f];
    }
    return 0;
}

/* ------------------------------------------------------------------------------------ */
/* output format (segmentedSieve.C:645-677, 816-819, 763-791)                             */
/* ------------------------------------------------------------------------------------ */

/* OutputTags: " (prime)" [", "] | " (2^N)" [',' + setw(3-floor(log10 N)) " "] | [",         "] */
static int tag(const ffo_ctx* c, uint64_t term, int blanks, char* buf, size_t cap, size_t* pos)
{
    if (is_prime(c, term, NULL)) {
        if (append(buf, cap, pos, " (prime)")) return -1;
        if (blanks && append(buf, cap, pos, ", ")) return -1;
    } else if (((0 - term) & term) == term) {
        double p2 = floor(log((double)term) / log((double)2) + .5);
        if (append(buf, cap, pos, " (2^%.0f)", p2)) return -1;
        if (blanks) {
            int w = (int)(3 - floor(log10(p2)));
            if (append(buf, cap, pos, ",%*s", w, " ")) return -1;
        }
    } else if (blanks) {
        if (append(buf, cap, pos, ",         ")) return -1;
    }
    return 0;
}

int ffo_format_line(const ffo_ctx* c, uint32_t count, uint32_t sum, uint32_t low, uint32_t high,
                    char* buf, size_t cap)
{
    size_t pos = 0;
    if (append(buf, cap, &pos, "%7u) sum =%9u, product =%16llu,  low term =%9u", count, sum,
               (unsigned long long)low * high, low))
        return -1;
    if (tag(c, low, 1, buf, cap, &pos)) return -1;
    if (append(buf, cap, &pos, "high term =%9u", high)) return -1;
    if (tag(c, high, 0, buf, cap, &pos)) return -1;
    if (append(buf, cap, &pos, "\n")) return -1;
    return (int)pos;
}

void ffo_free(void* p) { free(p); }

typedef struct {
    char* p;
    size_t n, cap;
} sbuf;

static int sb_put(sbuf* b, const char* s, size_t n)
{
    if (b->n + n + 1 > b->cap) {
        size_t nc = b->cap ? b->cap : 4096;
        while (nc < b->n + n + 1) nc *= 2;
        char* q = realloc(b->p, nc);
        if (!q) return -1;
        b->p = q;
        b->cap = nc;
    }
    memcpy(b->p + b->n, s, n);
    b->n += n;
    b->p[b->n] = 0;
    return 0;
}

/* The text ff_seg prints for one argument list, from per-sum records: the header, the
 * solution lines of the schedule in emission order (segmentedSieve.C:763-791, 816-819) and
 * the two timing lines normalised to "N". rec[(s - rec_lo)/2] = low<<32 | high or 0 for the
 * odd sums rec_lo, rec_lo+2, ...; every sum of the schedule must be covered. */
char* ffo_emit(const ffo_ctx* c, int nargs, int32_t a1, int32_t a2, const uint64_t* rec,
               uint32_t rec_lo, uint64_t nrec, size_t* len)
{
    uint32_t ss, sl;
    ffo_parse_args(nargs, a1, a2, &ss, &sl);
    ffo_geometry g;
    char hdr[2048];
    int hn = ffo_geometry_headers(ss, sl, &g, hdr, sizeof hdr);
    if (hn < 0 || g.too_big) return NULL;
    int cap = 4 * (int)FFO_THREADS + 8;
    uint32_t firsts[4 * FFO_THREADS + 8], lasts[4 * FFO_THREADS + 8];
    int nr = ffo_schedule(ss, sl, g.max_prime_map_value, FFO_THREADS, firsts, lasts, cap);
    if (nr < 0) return NULL;
    const uint64_t rec_hi = (uint64_t)rec_lo + 2 * (nrec ? nrec - 1 : 0);
    for (int r = 0; r < nr; ++r) {
        uint32_t f = firsts[r] | 1u;
        if (f > lasts[r]) continue;
        uint32_t l = lasts[r] - !(lasts[r] & 1);
        if (!rec || nrec == 0 || !(rec_lo & 1) || f < rec_lo || l > rec_hi) return NULL;
    }
    sbuf out = {0};
    sb_put(&out, hdr, (size_t)hn);
    uint32_t count = 0;
    char line[256];
    for (int r = 0; r < nr; ++r) {
        for (uint32_t s = firsts[r] | 1u; s <= lasts[r]; s += 2) {
            uint64_t v = rec[(s - rec_lo) / 2];
            if (!v) continue;
            int n = ffo_format_line(c, ++count, s, (uint32_t)(v >> 32), (uint32_t)v, line,
                                    sizeof line);
            sb_put(&out, line, (size_t)n);
        }
    }
    const char* tail = "Prime time: N \xce\xbcs\nFreudenthal time: N \xce\xbcs\n";
    sb_put(&out, tail, strlen(tail));
    if (len) *len = out.n;
    return out.p;
}

char* ffo_run(int nargs, int32_t a1, int32_t a2, uint64_t map_bound, int nthreads, size_t* len,
              ffo_counters* k)
{
    uint32_t ss, sl;
    ffo_parse_args(nargs, a1, a2, &ss, &sl);
    ffo_geometry g;
    char hdr[2048];
    int hn = ffo_geometry_headers(ss, sl, &g, hdr, sizeof hdr);
    if (hn < 0 || g.too_big) return NULL;
    int cap = 4 * (int)FFO_THREADS + 8;
    uint32_t firsts[4 * FFO_THREADS + 8], lasts[4 * FFO_THREADS + 8];
    int nr = ffo_schedule(ss, sl, g.max_prime_map_value, FFO_THREADS, firsts, lasts, cap);
    if (nr < 0) return NULL;
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    for (int r = 0; r < nr; ++r) {
        uint32_t f = firsts[r] | 1u;
        if (f > lasts[r]) continue;
        if (f < lo) lo = f;
        if (lasts[r] > hi) hi = lasts[r];
    }
    ffo_ctx* c = ffo_create(hi > sl ? hi : sl, map_bound ? map_bound : g.max_prime_map_value,
                            nthreads);
    if (!c) return NULL;
    uint64_t* rec = NULL;
    uint64_t nrec = 0;
    if (lo <= hi) {
        hi -= !(hi & 1);   /* last odd sum */
        nrec = ((uint64_t)hi - lo) / 2 + 1;
        rec = calloc(nrec, sizeof(uint64_t));
        ffo_eval_range(c, lo, hi, rec, nthreads, k);
    } else {
        lo = 1;
    }
    char* out = NULL;
    if (nrec) {
        out = ffo_emit(c, nargs, a1, a2, rec, lo, nrec, len);
    } else {
        uint64_t dummy = 0;   /* no sums in the schedule: header and timing lines only */
        out = ffo_emit(c, nargs, a1, a2, &dummy, 1, 1, len);
    }
    free(rec);
    ffo_destroy(c);
    return out;
}
