/* Multithreaded text I/O of .n data (values one per line, or any whitespace
 * between them): the bytes read and written are those of one strtod and one
 * fprintf("%.*e\n") per value, in order, for any OpenMP thread count. */
#ifndef PFC_NIO_H
#define PFC_NIO_H

#include <stddef.h>
#include <stdio.h>

/* The first n whitespace-separated numbers of [q, e) into out. Returns 0, or 1
 * when fewer than n numbers precede the first token that is not a number (or
 * the end). Text after the first n numbers is not looked at. */
int nio_parse_values(const char* q, const char* e, double* out, size_t n);

/* fprintf(f, "%.*e\n", prec, v[i]) for i = 0 .. n-1. */
void nio_write_values(FILE* f, int prec, const double* v, size_t n);

/* fprintf(f, "%.*e %.*e\n", prec, a[i], prec, b[i]) for i = 0 .. n-1. */
void nio_write_pairs(FILE* f, int prec, const double* a, const double* b, size_t n);

/* Whole file into a NUL-terminated buffer (free() it); NULL if unreadable. */
char* nio_slurp(const char* path, size_t* len);

#endif
