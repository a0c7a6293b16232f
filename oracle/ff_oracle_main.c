/*
 * ff_oracle_main.c -- command-line front end of the CPU restatement (checker only).
 *
 *   ff_oracle [--map-bound B] [--threads T] [--counters] [<sumStart>] [<sumLimit>]
 *
 * Prints what ff_seg prints for the same positional arguments (segmentedSieve.C:829-925),
 * with the two timing lines normalised to "N". --map-bound limits the bitmap to values
 * <= B (Miller-Rabin above it); --counters adds the instrumented work totals on stderr.
 */
#include "ff_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int main(int argc, char** argv)
{
    uint64_t bound = 0;
    int threads = 8, counters = 0, nargs = 0;
    int32_t a[2] = {0, 0};
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "--map-bound") && i + 1 < argc) {
            bound = strtoull(argv[++i], NULL, 10);
        } else if (!strcmp(argv[i], "--threads") && i + 1 < argc) {
            threads = atoi(argv[++i]);
        } else if (!strcmp(argv[i], "--counters")) {
            counters = 1;
        } else if (nargs < 2) {
            a[nargs++] = atoi(argv[i]);
        } else {
            fprintf(stderr, "ff_oracle: unexpected argument '%s'\n", argv[i]);
            return 2;
        }
    }
    ffo_counters k;
    memset(&k, 0, sizeof k);
    size_t len = 0;
    char* out = ffo_run(nargs, a[0], a[1], bound, threads, &len, &k);
    if (!out) {
        fprintf(stderr, "ff_oracle: range outside what the reference can run\n");
        return 1;
    }
    fwrite(out, 1, len, stdout);
    ffo_free(out);
    if (counters)
        fprintf(stderr,
                "sums %llu map_probes %llu mr_calls %llu mr_mulmods %llu splits %llu "
                "abop_calls %llu trial_steps %llu divisors %llu errors %llu\n",
                (unsigned long long)k.sums, (unsigned long long)k.map_probes,
                (unsigned long long)k.mr_calls, (unsigned long long)k.mr_mulmods,
                (unsigned long long)k.splits, (unsigned long long)k.abop_calls,
                (unsigned long long)k.trial_steps, (unsigned long long)k.divisors,
                (unsigned long long)k.errors);
    return k.errors ? 3 : 0;
}
