// ff_sieve_main.cpp -- the `ff_sieve [<sumStart>] [<sumLimit>]` command (reference CLI:
// source/main.cpp:577-598 with ff_seg's positional semantics, reference/segmentedSieve.C:
// 844-855). stdout carries exactly what ff_seg prints; stderr carries diagnostics.
// Return code 0 on success, 1 on any error.
//
// `ff_sieve --dump-map <file> [<sumStart>] [<sumLimit>]` is ff_seg's sieve-only test option
// (reference/segmentedSieve.C:830-839, 883-897): the header lines on stdout, the prime map
// (Prime::PrimeMapSize() bytes) written to <file>, no search; its messages and exit codes
// are ff_seg's (-6 no file argument or file not writable, -7 write failed). The flags that
// the reference's scripts/verify.sh passes to its GPU binary (--devices nvidia, --gpu-search,
// --dump-map <file> in any position) are accepted, so that harness runs unchanged.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ffb200.h"

static void usage()
{
    std::fprintf(stderr,
                 "usage: ff_sieve [--device N] [--devices nvidia] [--gpu-search]\n"
                 "                [--dump-map <file>] [<sumStart>] [<sumLimit>]\n"
                 "  one positional argument: sums 5..<sumLimit>; none: 5..2627\n");
}

static int dump_map(int device, const char* file, int nargs, const int32_t* a)
{
    uint8_t* map = nullptr;
    uint64_t bytes = 0;
    char hdr[4096];
    if (ffb_map_dump(device, nargs, a[0], a[1], &map, &bytes, hdr, sizeof hdr) != 0) return 1;
    std::fputs(hdr, stdout);
    std::fflush(stdout);
    FILE* f = std::fopen(file, "wb");
    if (!f) {
        std::printf("Cannot open dump file '%s' for writing.\n", file);
        ffb_free(map);
        return -6;
    }
    const bool ok = std::fwrite(map, 1, bytes, f) == bytes;
    ffb_free(map);
    if (std::fclose(f) != 0 || !ok) {
        std::printf("Failed to write dump file '%s'.\n", file);
        return -7;
    }
    return 0;
}

int main(int argc, char** argv)
{
    int device = 0, nargs = 0;
    int32_t a[2] = {0, 0};
    if (argc > 1 && !std::strcmp(argv[1], "--dump-map")) {
        if (argc < 3) {
            std::printf("--dump-map requires a file argument.\n");
            return -6;
        }
        const char* file = argv[2];
        for (int i = 3; i < argc; ++i) {
            if (!std::strcmp(argv[i], "--device") && i + 1 < argc) device = std::atoi(argv[++i]);
            else if (nargs < 2) a[nargs++] = std::atoi(argv[i]);
        }
        return dump_map(device, file, nargs, a);
    }
    const char* dump = nullptr;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--device") && i + 1 < argc) {
            device = std::atoi(argv[++i]);
        } else if (!std::strcmp(argv[i], "--devices") && i + 1 < argc) {
            // the reference's vendor filter (source/config.cpp:353-363): only CUDA devices here
            const char* b = argv[++i];
            if (std::strcmp(b, "nvidia") && std::strcmp(b, "NVIDIA")) {
                std::fprintf(stderr, "ff_sieve: --devices %s: this build runs on NVIDIA "
                             "(sm_100a) devices only\n", b);
                return 1;
            }
        } else if (!std::strcmp(argv[i], "--gpu-search")) {
            // the reference's switch to its GPU search (source/config.cpp:375-378): the
            // search always runs on the GPU here
        } else if (!std::strcmp(argv[i], "--dump-map") && i + 1 < argc) {
            dump = argv[++i];  // ff_sieve's form (source/config.cpp:365-369): any position
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
    if (dump) return dump_map(device, dump, nargs, a);
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
