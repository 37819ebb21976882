/*
 * opt_parser.h - CLI list and range parsing.
 *
 * Drop-in for the reference's include/opt_parser.h: positive integers,
 * comma-separated lists and start:end[:step] ranges, sorted and made unique
 * (reference src/opt_parser.c:68-201).
 */
#ifndef OPT_PARSER_H
#define OPT_PARSER_H

#include <stddef.h>

typedef struct
{
    int *values;
    size_t size;
    size_t capacity;
} OptIntList;

void opt_int_list_init(OptIntList *list);
void opt_int_list_free(OptIntList *list);
/* Appends a positive value; returns 0, or -1 for value <= 0 / OOM. */
int opt_int_list_append(OptIntList *list, int value);
/* Sorts ascending and removes duplicates in place. */
void opt_int_list_sort_unique(OptIntList *list);
/* Decimal string -> positive int in [1, INT_MAX]; returns 0 or -1. */
int opt_parse_positive_int(const char *text, int *out);
/* "1,4,8" or "1:16:2" (and mixes) -> sorted unique list; returns 0 or -1
 * (with a message naming `label` on stderr). */
int opt_parse_range_list(const char *spec, OptIntList *list, const char *label);

#endif /* OPT_PARSER_H */
