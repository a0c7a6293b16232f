// ff_sieve_main.cpp -- the `ff_sieve [<sumStart>] [<sumLimit>]` command (reference CLI:
// source/main.cpp:577-598 with ff_seg's positional semantics, reference/segmentedSieve.C:
// 844-855). stdout carries exactly what ff_seg prints; stderr carries diagnostics.
// Return code 0 on success, 1 on any error.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ffb200.h"

static void usage()
{
    std::fprintf(stderr,
                 "usage: ff_sieve [--device N] [<sumStart>] [<sumLimit>]\n"
                 "  one positional argument: sums 5..<sumLimit>; none: 5..2627\n");
}

int main(int argc, char** argv)
{
    int device = 0, nargs = 0;
    int32_t a[2] = {0, 0};
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else if (!std::strcmp(argv[i], "--help") || !std::strcmp(argv[i], "-h")) {
            usage();
            return 0;
        } else if (argv[i][0] == '-' && argv[i][1] == '-') {
            std::fprintf(stderr, "ff_sieve: unknown option '%s'\n", argv[i]);
            usage();
            return 1;
        } else if (nargs < 2) {
            a[nargs++] = std::atoi(argv[i]);
        } else {
            usage();
            return 1;
        }
    }
    FfbContext* ctx = ffb_context_create(device);
    if (!ctx) {
        std::fprintf(stderr, "ff_sieve: no usable CUDA device %d\n", device);
        return 1;
    }
    char* text = nullptr;
    size_t len = 0;
    const int rc = ffb_run(ctx, nargs, a[0], a[1], &text, &len);
    ffb_context_destroy(ctx);
    if (rc) return 1;
    std::fwrite(text, 1, len, stdout);
    ffb_free(text);
    return 0;
}
