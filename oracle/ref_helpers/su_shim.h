/*
 * Stand-ins for the few Seismic Unix (SU/CWP) declarations that the
 * reference's CPU helper files use (alloc/free wrappers, the `complex` struct,
 * PI, warn/err).  SU itself is not vendored in the reference tree.  Only the
 * arithmetic-free plumbing is supplied here; every numeric line that the
 * golden vectors exercise is the reference's own, compiled from the
 * reference tree where it lies.  Used only to generate tests/golden fixtures.
 */
#pragma once
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define PI 3.141592653589793
typedef struct { float r, i; } complex;
static float *alloc1float(size_t n) { return (float *)calloc(n, sizeof(float)); }
static void free1float(float *p) { free(p); }
static int *alloc1int(size_t n) { return (int *)calloc(n, sizeof(int)); }
static void free1int(int *p) { free(p); }
static float **alloc2float(size_t n1, size_t n2)
{
    float **p = (float **)malloc(n2 * sizeof(float *));
    float *d = (float *)calloc(n1 * n2, sizeof(float));
    for (size_t i = 0; i < n2; i++) p[i] = d + i * n1;
    return p;
}
static void free2float(float **p) { free(p[0]); free(p); }
static complex **alloc2complex(size_t n1, size_t n2)
{
    complex **p = (complex **)malloc(n2 * sizeof(complex *));
    complex *d = (complex *)calloc(n1 * n2, sizeof(complex));
    for (size_t i = 0; i < n2; i++) p[i] = d + i * n1;
    return p;
}
static void free2complex(complex **p) { free(p[0]); free(p); }
static void warn(const char *f, ...) { (void)f; }
static void err(const char *f, ...) { (void)f; exit(1); }
