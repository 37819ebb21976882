/*
 * results_writer.h - the benchmark's CSV file.
 *
 * Drop-in for the reference's include/results_writer.h: one column per
 * configuration, one row per run, values printed "%.6f"; appending to an
 * existing column adds rows below the longest column, a new column is padded
 * with empty cells (reference src/results_writer.c:301-582).
 */
#ifndef RESULTS_WRITER_H
#define RESULTS_WRITER_H

#include <stddef.h>

typedef enum
{
    RESULTS_WRITER_OK = 0,
    RESULTS_WRITER_IO_ERROR = -1,
    RESULTS_WRITER_MEMORY_ERROR = -2,
    RESULTS_WRITER_INVALID_ARGS = -3
} results_writer_status;

results_writer_status append_times_column(const char *filename, const char *column_name,
                                          const double *values, size_t count);
/* mkdir -p; 0 or -1 (errno set). */
int results_writer_ensure_directory(const char *path);
/* dest = dir + "/" + file (no doubled slash); 0 or -1. */
int results_writer_join_path(char *dest, size_t dest_size, const char *dir, const char *file);
/* Base name of matrix_path without its last extension ("graph" if empty). */
int results_writer_matrix_stem(const char *matrix_path, char *dest, size_t dest_size);
/* <output_dir>/<prefix>_<stem>.csv */
int results_writer_build_results_path(char *dest, size_t dest_size, const char *output_dir,
                                      const char *prefix, const char *matrix_path);

#endif /* RESULTS_WRITER_H */
