/*
 * mpi_cc_benchmark - the reference's benchmark driver on one B200.
 *
 * Same flags (-c/-e/-r/-o/-t/-h, src/mpi_cc_benchmark.c:17-29), sweep
 * (chunk x exchange x runs, :192-219), timed region (one
 * compute_connected_components_mpi_advanced call, :206-212) and CSV
 * (<out>/results_mpi_<stem>.csv, one column chunk_<c>_exchange_<e>, "%.6f"
 * seconds per run, :221-237).  The partition count that mpirun -np gives
 * the reference comes from -p (or CCB200_PARTITIONS).  Additions: -L FILE
 * writes the labels of the last run (raw uint32), -q silences the solver's
 * summary lines, -v prints its phase lines.
 */
#include <errno.h>
#include <getopt.h>
#include <inttypes.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "cc_mpi.h"
#include "graph_dist.h"
#include "opt_parser.h"
#include "results_writer.h"
#include "runtime_utils.h"

static void usage(const char *prog)
{
    fprintf(stderr,
            "Usage: %s [OPTIONS] <matrix-file-path>\n\n"
            "Options:\n"
            "  -c, --chunk-size SPEC       Chunk size list/range\n"
            "  -e, --exchange SPEC         Exchange interval list/range\n"
            "  -r, --runs N                Runs per configuration (default 1)\n"
            "  -o, --output DIR            Output directory (default 'results')\n"
            "  -t, --threads N             Host threads per partition (default: all cores)\n"
            "  -p, --partitions N          Partitions, as mpirun -np (default 1 or\n"
            "                              $CCB200_PARTITIONS)\n"
            "  -L, --labels FILE           Write the last run's labels (uint32)\n"
            "  -q, --quiet                 No solver summary lines\n"
            "  -v, --verbose               Solver phase lines\n"
            "  -h, --help                  Show help message\n",
            prog);
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int main(int argc, char **argv)
{
    const char *chunk_spec = "2048", *exchange_spec = "1", *output_dir = "results";
    const char *labels_path = NULL;
    int runs = 1, threads_opt = 0, parts = 0, verbose = 1;

    const struct option long_opts[] = {{"chunk-size", required_argument, NULL, 'c'},
                                       {"exchange", required_argument, NULL, 'e'},
                                       {"runs", required_argument, NULL, 'r'},
                                       {"output", required_argument, NULL, 'o'},
                                       {"threads", required_argument, NULL, 't'},
                                       {"partitions", required_argument, NULL, 'p'},
                                       {"labels", required_argument, NULL, 'L'},
                                       {"quiet", no_argument, NULL, 'q'},
                                       {"verbose", no_argument, NULL, 'v'},
                                       {"help", no_argument, NULL, 'h'},
                                       {NULL, 0, NULL, 0}};
    int opt, idx;
    while ((opt = getopt_long(argc, argv, "c:e:r:o:t:p:L:qvh", long_opts, &idx)) != -1) {
        switch (opt) {
        case 'c':
            chunk_spec = optarg;
            break;
        case 'e':
            exchange_spec = optarg;
            break;
        case 'r':
            if (opt_parse_positive_int(optarg, &runs) != 0) {
                fprintf(stderr, "Invalid runs: %s\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'o':
            output_dir = optarg;
            break;
        case 't':
            if (opt_parse_positive_int(optarg, &threads_opt) != 0) {
                fprintf(stderr, "Invalid threads: %s\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'p':
            if (opt_parse_positive_int(optarg, &parts) != 0 || parts > CCGPU_MAX_PARTS) {
                fprintf(stderr, "Invalid partitions: %s\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'L':
            labels_path = optarg;
            break;
        case 'q':
            verbose = 0;
            break;
        case 'v':
            verbose = 2;
            break;
        case 'h':
            usage(argv[0]);
            return EXIT_SUCCESS;
        default:
            usage(argv[0]);
            return EXIT_FAILURE;
        }
    }
    if (optind >= argc) {
        fprintf(stderr, "Missing matrix file path.\n");
        usage(argv[0]);
        return EXIT_FAILURE;
    }
    const char *matrix_path = argv[optind];

    int threads = threads_opt > 0 ? threads_opt : runtime_default_threads();
    cc_mpi_set_num_threads(threads < 1 ? 1 : threads);
    if (parts > 0 && cc_group_set_world_size(parts) != 0) {
        fprintf(stderr, "Invalid partitions: %d\n", parts);
        return EXIT_FAILURE;
    }
    MPI_Comm comm = cc_group_world();
    cc_group_set_verbose(comm, verbose);
    if (ccgpu_device_check() != CCGPU_OK) {
        fprintf(stderr, "%s\n", ccgpu_last_error());
        return EXIT_FAILURE;
    }
    printf("CC B200 Benchmark (partitions=%d, host threads=%d)\n", cc_group_size(comm),
           cc_mpi_get_num_threads());

    if (results_writer_ensure_directory(output_dir) != 0) {
        fprintf(stderr, "Failed to create output directory '%s': %s\n", output_dir,
                strerror(errno));
        return EXIT_FAILURE;
    }
    OptIntList chunks, exchanges;
    opt_int_list_init(&chunks);
    opt_int_list_init(&exchanges);
    if (opt_parse_range_list(chunk_spec, &chunks, "chunk sizes") != 0) {
        fprintf(stderr, "Invalid chunk-size specification.\n");
        return EXIT_FAILURE;
    }
    if (opt_parse_range_list(exchange_spec, &exchanges, "exchange intervals") != 0) {
        fprintf(stderr, "Invalid exchange interval specification.\n");
        opt_int_list_free(&chunks);
        return EXIT_FAILURE;
    }
    char results_path[PATH_MAX];
    if (results_writer_build_results_path(results_path, sizeof(results_path), output_dir,
                                          "results_mpi", matrix_path) != 0) {
        fprintf(stderr, "Failed to build results path.\n");
        return EXIT_FAILURE;
    }
    printf("Saving results to: %s\n", results_path);

    double *run_times = (double *)malloc((size_t)runs * sizeof(double));
    if (!run_times) {
        fprintf(stderr, "Memory allocation failed (run_times).\n");
        return EXIT_FAILURE;
    }
    DistCSRGraph Gd;
    double t0 = now_s();
    int rc = load_dist_csr_from_file(matrix_path, 1, 1, 1, &Gd, comm); /* :178 */
    double t1 = now_s();
    if (rc != 0) {
        fprintf(stderr, "Error loading graph.\n");
        return EXIT_FAILURE;
    }
    printf("Graph loaded (n=%" PRIu32 ", m=%" PRIu64 ") in %.6f seconds.\n", Gd.n_global,
           Gd.m_global, t1 - t0);
    uint32_t *labels = NULL;
    if (labels_path) {
        labels = (uint32_t *)malloc((size_t)(Gd.n_global ? Gd.n_global : 1) * sizeof(uint32_t));
        if (!labels) {
            fprintf(stderr, "Memory allocation failed (labels).\n");
            return EXIT_FAILURE;
        }
    }

    for (size_t ci = 0; ci < chunks.size; ++ci) {
        int chunk = chunks.values[ci];
        for (size_t ei = 0; ei < exchanges.size; ++ei) {
            int exchange = exchanges.values[ei];
            printf("\n=== Testing chunk=%d, exchange=%d (%d run%s) ===\n", chunk, exchange, runs,
                   runs == 1 ? "" : "s");
            for (int r = 0; r < runs; ++r) {
                double a = now_s();
                compute_connected_components_mpi_advanced(&Gd, labels, chunk, exchange, comm);
                double b = now_s();
                run_times[r] = b - a;
                printf("Run %d: %.6f seconds\n", r + 1, run_times[r]);
            }
            char colname[128];
            snprintf(colname, sizeof(colname), "chunk_%d_exchange_%d", chunk, exchange);
            results_writer_status st =
                append_times_column(results_path, colname, run_times, (size_t)runs);
            if (st != RESULTS_WRITER_OK)
                fprintf(stderr, "Warning: CSV update failed (%d) for %s\n", st, colname);
            printf("Saved column '%s' to %s\n", colname, results_path);
        }
    }
    if (labels_path) {
        FILE *f = fopen(labels_path, "wb");
        if (!f || fwrite(labels, sizeof(uint32_t), Gd.n_global, f) != Gd.n_global) {
            fprintf(stderr, "Failed to write labels to %s\n", labels_path);
            if (f)
                fclose(f);
            return EXIT_FAILURE;
        }
        fclose(f);
    }
    free(labels);
    free_dist_csr(&Gd);
    free(run_times);
    opt_int_list_free(&chunks);
    opt_int_list_free(&exchanges);
    printf("\nAll tests completed.\n");
    return EXIT_SUCCESS;
}
