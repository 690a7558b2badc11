// cli_main.cpp -- the per-app command line of the reference, on libgft.
//
//   bfs  [-q] [-g gpunum] [-o output-file] [-l] [-s startNode] graph-file
//   sssp [-q] [-g gpunum] [-o output-file] [-l] [-d delta] [-s startNode] graph-file
//   cc   [-q] [-g gpunum] [-o output-file] graph-file
//   pr   [-q] [-g gpunum] [-o output-file] [-n] [-t top_ranks] [-x max_iterations] graph-file
//   mis  [-q] [-g gpunum] [-o output-file] graph-file
//
// Same options, same stdout/stderr lines and same output file as the
// reference driver (skelapp/skel.cu:37-151 with apps/bfs/support.cu:5-45,
// apps/sssp/support.cu:6-53, apps/cc/support.cu:3-36, apps/pr/support.cu:
// 15-104 and apps/mis/support.cu:1-40; cc prints the reference's
// "components: N" line, apps/cc/kernel.cu:719, pr its "PR took N iterations"
// and "sum: S (N)" lines, and mis its "Total steps: N" line,
// apps/mis/kernel.cu:231).  CC labels are
// the smallest vertex id of each component, where the reference's are
// whichever roots its racy hooks leave: the partition is the same.  The traversal runs through the C ABI.  `-l`
// (the reference's host-driven load balancer, apps/bfs/kernel.cu:286-311) is
// accepted for compatibility; this engine always balances per vertex inside
// its persistent kernel.  Errors are reported and turned into a non-zero
// exit code instead of exit(1) deep inside the library.
//
// Two additions for large results and graphs: `-b file` writes the result
// array as a binary dump (gft_write_node_data), and an -o file name ending
// in ".gz" gets the same text gzip-compressed (gft_write_output_gz; bfs and
// sssp).  Every app but cc reads the .gr file straight into device memory
// (gft_graph_load_gr); cc's output lists every edge, so it keeps a host copy.
#include <getopt.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <vector>

#include "gft.h"

// The app this binary is: 0 bfs, 1 sssp, 2 cc, 3 pr, 4 mis (set by the build).
#ifndef GFT_CLI_APP
#define GFT_CLI_APP 0
#endif
#define GFT_CLI_SSSP (GFT_CLI_APP == 1)
#define GFT_CLI_CC (GFT_CLI_APP == 2)
#define GFT_CLI_PR (GFT_CLI_APP == 3)
#define GFT_CLI_MIS (GFT_CLI_APP == 4)
#define GFT_CLI_NO_SOURCE (GFT_CLI_CC || GFT_CLI_PR || GFT_CLI_MIS)

static const char *kAppOpts = GFT_CLI_PR ? "nt:x:" : (GFT_CLI_CC || GFT_CLI_MIS) ? "" : GFT_CLI_SSSP ? "ls:d:" : "ls:";
static const char *kAppUsage = GFT_CLI_PR   ? "[-n] [-t top_ranks] [-x max_iterations]"
                               : (GFT_CLI_CC || GFT_CLI_MIS) ? ""
                               : GFT_CLI_SSSP ? "[-l] [-d delta] [-s startNode]"
                                              : "[-l] [-s startNode]";
static const char *kAppArgsUsage =
    GFT_CLI_NO_SOURCE ? "" : "-l: enable thread block load balancer (by default false)";

static void usage(const char *argv0)
{
    fprintf(stderr, "usage: %s [-q] [-g gpunum] [-o output-file] [-b binary-dump] %s graph-file \n %s\n", argv0,
            kAppUsage, kAppArgsUsage);
}

static uint64_t now_ns()
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC_RAW, &ts);
    return (uint64_t)ts.tv_sec * 1000000000ull + ts.tv_nsec;
}

static int die(const char *what, gft_status s)
{
    fprintf(stderr, "%s: %s: %s\n", what, gft_status_string(s), gft_last_error());
    return 1;
}

int main(int argc, char **argv)
{
    if (argc == 1) {
        usage(argv[0]);
        return 1;
    }
    int quiet = 0, device = 0, start_node = 0, delta = 10000, no_print_rank = 0;
    uint32_t max_iterations = 0xFFFFFFFFu;
    const char *output = nullptr, *dump = nullptr;
    char opts[32];
    snprintf(opts, sizeof opts, "g:qo:b:%s", kAppOpts);
    int c;
    while ((c = getopt(argc, argv, opts)) != -1) {
        switch (c) {
        case 'q': quiet = 1; break;
        case 'o': output = optarg; break;
        case 'b': dump = optarg; break;
        case 'g': {
            char *end;
            device = (int)strtol(optarg, &end, 10);
            if (*end != '\0') {
                fprintf(stderr, "Invalid GPU device '%s'. An integer must be specified.\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        }
        case 's':
            start_node = atoi(optarg);
            if (start_node < 0) {
                fprintf(stderr, "start node must be >= 0\n");
                return EXIT_FAILURE;
            }
            break;
        case 'd':
            delta = atoi(optarg);
            if (delta <= 0) {
                fprintf(stderr, "delta must be > 0\n");
                return EXIT_FAILURE;
            }
            break;
        case 'l': break;
        case 'n': no_print_rank = 1; break;
        case 't': break;  // accepted: the reference's output ignores it (apps/pr/support.cu:83-94)
        case 'x': max_iterations = (uint32_t)strtoul(optarg, nullptr, 10); break;
        default: usage(argv[0]); return EXIT_FAILURE;
        }
    }
    if (optind >= argc) {
        usage(argv[0]);
        return EXIT_FAILURE;
    }
    const char *input = argv[optind];

    fprintf(stderr, "OPTIONS: gft engine (libgft %d, sm_100a %s)\n", gft_version(),
            GFT_CLI_MIS  ? "persistent round-based MIS"
            : GFT_CLI_PR ? "persistent residual-push PageRank" : GFT_CLI_CC ? "union-find CC"
            : GFT_CLI_SSSP ? "persistent near-far SSSP" : "persistent BFS");
    gft_csr h;
    memset(&h, 0, sizeof h);
    gft_graph *g = nullptr;
    gft_engine *e = nullptr;
    uint64_t t0 = now_ns();
    gft_status s;
    if (GFT_CLI_CC) {
        if ((s = gft_gr_read(input, &h)) != GFT_OK) return die("read", s);
        if ((s = gft_graph_upload(device, &h, nullptr, &g)) != GFT_OK) return die("upload", s);
    } else {
        if ((s = gft_graph_load_gr(device, input, nullptr, &g)) != GFT_OK) return die("read", s);
        int weighted = 0;
        gft_graph_info(g, &h.nnodes, &h.nedges, &weighted);
    }
    printf("nnodes=%u, nedges=%u.\n", h.nnodes, h.nedges);
    printf("read %s in %llu ms\n", input, (unsigned long long)((now_ns() - t0) / 1000000));
    if (!GFT_CLI_NO_SOURCE && (uint32_t)start_node >= h.nnodes) {
        fprintf(stderr, "start node %d out of range (%u nodes)\n", start_node, h.nnodes);
        gft_graph_free(g);
        gft_csr_free(&h);
        return EXIT_FAILURE;
    }
    if ((s = gft_engine_create(device, &e)) != GFT_OK) return die("engine", s);
    printf("Using GPU: %d\n", device);

    std::vector<int32_t> val(h.nnodes);
    gft_stats st;
    memset(&st, 0, sizeof st);
    uint64_t comps = 0;
    std::vector<float> rank(GFT_CLI_PR ? h.nnodes : 0);
    uint64_t k0 = now_ns();
    if (GFT_CLI_MIS) {
        s = gft_mis_host(e, g, val.data(), 0, nullptr, nullptr, &st);
    } else if (GFT_CLI_PR) {
        s = gft_pr_host(e, g, rank.data(), max_iterations, nullptr, nullptr, &st);
    } else if (GFT_CLI_CC) {
        s = gft_cc_host(e, g, val.data(), nullptr, nullptr, &st, &comps);
    } else if (GFT_CLI_SSSP) {
        printf("delta: %d\n", delta);
        s = gft_sssp_host(e, g, (uint32_t)start_node, delta, val.data(), nullptr, nullptr, nullptr, &st);
    } else {
        s = gft_bfs_host(e, g, (uint32_t)start_node, val.data(), nullptr, nullptr, nullptr, &st);
    }
    uint64_t k1 = now_ns();
    if (s != GFT_OK)
        return die(GFT_CLI_MIS ? "mis" : GFT_CLI_PR ? "pr" : GFT_CLI_CC ? "cc" : GFT_CLI_SSSP ? "sssp" : "bfs", s);
    if (GFT_CLI_MIS) printf("Total steps: %u\n", st.levels);
    if (GFT_CLI_PR) printf("PR took %u iterations\n", st.levels);
    if (GFT_CLI_SSSP) printf("iterations: %u\n", st.levels);
    if (GFT_CLI_CC) printf("components: %llu\n", (unsigned long long)comps);
    printf("gg_main %llu %llu\n", (unsigned long long)k0, (unsigned long long)k1);
    fprintf(stderr, "Total time: %llu ms\n", (unsigned long long)((k1 - k0) / 1000000));
    fprintf(stderr, "Total time: %llu ns\n", (unsigned long long)(k1 - k0));
    fprintf(stderr, "Kernel time: %.3f ms (%u levels/phases, %u grid iterations)\n", st.kernel_ms, st.levels,
            st.iterations);
    int rc = 0;
    if (GFT_CLI_PR && !quiet) {  // apps/pr/support.cu:56-65: a float sum in node order
        fprintf(stderr, "Calculating sum ...\n");
        float sum = 0;
        for (uint32_t i = 0; i < h.nnodes; i++) sum += rank[i];
        fprintf(stdout, "sum: %f (%d)\n", (double)sum, (int)h.nnodes);
    }
    if (!quiet && output) {
        if (GFT_CLI_PR && no_print_rank) {
            FILE *f = strcmp(output, "-") == 0 ? stdout : fopen(output, "w");
            if (!f) {
                fprintf(stderr, "output: cannot open %s\n", output);
                rc = 1;
            } else {
                for (uint32_t i = 0; i < h.nnodes; i++) fprintf(f, "%d\n", (int)i);
                if (f != stdout) fclose(f);
            }
            s = GFT_OK;
        } else if (GFT_CLI_PR) {
            s = gft_write_pr_output(output, h.nnodes, rank.data());
        } else if (GFT_CLI_MIS) {
            s = gft_write_mis_output(output, h.nnodes, val.data());
        } else if (GFT_CLI_CC) {
            s = gft_write_cc_output(output, &h, val.data());
        } else {
            const size_t len = strlen(output);
            s = len > 3 && strcmp(output + len - 3, ".gz") == 0 ? gft_write_output_gz(output, h.nnodes, val.data(), 1)
                                                                : gft_write_output(output, h.nnodes, val.data());
        }
        if (s != GFT_OK) rc = die("output", s);
    }
    if (!quiet && dump) {
        s = GFT_CLI_PR ? gft_write_node_data(dump, h.nnodes, rank.data(), GFT_ELEM_F32)
                       : gft_write_node_data(dump, h.nnodes, val.data(), GFT_ELEM_I32);
        if (s != GFT_OK) rc = die("binary dump", s);
    }
    gft_engine_destroy(e);
    gft_graph_free(g);
    gft_csr_free(&h);
    return rc;
}
