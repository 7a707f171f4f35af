/*
 * ref_print_wrap.c -- link-time print hook for the reference LULESH builds.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is linked (with GNU ld --wrap) into
 * the binaries that oracle/Makefile builds from the UNMODIFIED reference
 * sources into oracle/_ref/.  It changes nothing in the reference's
 * arithmetic: it only widens two print formats so the oracle can compare
 * at full double precision instead of 7 significant digits:
 *
 *   "%12.6e"  ->  "%.17e"   Final Origin Energy and the symmetry block
 *                           (LULESH/cuda/src/lulesh.cu:4710,4734-4736;
 *                            LULESH/omp_4.0/lulesh-util.cc:193-219)
 *   "%.10f"   ->  "%.17e"   xyz.asc node coordinates
 *                           (LULESH/cuda/src/lulesh.cu:4598-4600)
 *
 * Field positions of the awk-parsed lines do not change (the number is still
 * one whitespace-free token), so `awk '{print $5}'` on the energy line
 * (LULESH/run_lulesh_verify.sbatch:65) still works.
 */
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

static const char *widen(const char *fmt, char *buf, size_t cap)
{
    static const char *from[2] = {"%12.6e", "%.10f"};
    static const char *to = "%.17e";
    size_t o = 0;
    const char *p = fmt;
    int changed = 0;
    while (*p && o + 8 < cap) {
        int hit = 0;
        for (int k = 0; k < 2; ++k) {
            size_t n = strlen(from[k]);
            if (strncmp(p, from[k], n) == 0) {
                memcpy(buf + o, to, strlen(to));
                o += strlen(to);
                p += n;
                hit = 1;
                changed = 1;
                break;
            }
        }
        if (!hit) buf[o++] = *p++;
    }
    if (*p) return fmt; /* too long: leave untouched */
    buf[o] = '\0';
    return changed ? buf : fmt;
}

int __real_printf(const char *fmt, ...);
int __real_fprintf(FILE *f, const char *fmt, ...);

int __wrap_printf(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    int r = vprintf(widen(fmt, buf, sizeof buf), ap);
    va_end(ap);
    return r;
}

int __wrap___printf_chk(int flag, const char *fmt, ...)
{
    (void)flag;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    int r = vprintf(widen(fmt, buf, sizeof buf), ap);
    va_end(ap);
    return r;
}

int __wrap_fprintf(FILE *f, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    int r = vfprintf(f, widen(fmt, buf, sizeof buf), ap);
    va_end(ap);
    return r;
}

int __wrap___fprintf_chk(FILE *f, int flag, const char *fmt, ...)
{
    (void)flag;
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    int r = vfprintf(f, widen(fmt, buf, sizeof buf), ap);
    va_end(ap);
    return r;
}
