/* Stubs for the reference CPU build (test infrastructure only).
 * - CHOLMOD is not installed: the Cholesky back-substitution path
 *   (tomo.alg=0 / fit.alg=0) is off the CG path this build exercises, so every
 *   entry point of math/chol.h aborts if it is ever reached.
 * - maosref_siglist backs the sys_siglist name mapped in compat.h. */
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

const char *maosref_siglist[65];
__attribute__((constructor)) static void maosref_fill_siglist(void) {
    for (int i = 0; i < 65; i++) maosref_siglist[i] = strsignal(i);
}

#define CHOL_STUB(name) \
    void name(void) { fprintf(stderr, "reference build: %s needs CHOLMOD (not built)\n", #name); abort(); }
CHOL_STUB(chol_factorize)
CHOL_STUB(chol_solve)
CHOL_STUB(chol_spsolve)
CHOL_STUB(chol_free_do)
CHOL_STUB(chol_save)
CHOL_STUB(chol_read)
CHOL_STUB(chol_convert)
CHOL_STUB(chol_solve_lower)
CHOL_STUB(chol_solve_upper)

/* sys/mem.c routes every allocation through function pointers that its own
 * constructor fills in.  Inside one shared library the order of the
 * reference's constructors is the link order, and some run before mem.c's and
 * allocate; fill the pointers first, with libc's allocator. */
extern void *(*calloc_default)(size_t, size_t);
extern void *(*malloc_default)(size_t);
extern void *(*realloc_default)(void *, size_t);
extern void (*free_default)(void *);
__attribute__((constructor(101))) static void maosref_early_alloc(void) {
    calloc_default = calloc;
    malloc_default = malloc;
    realloc_default = realloc;
    free_default = free;
}

/* sys/process.c creates $HOME/.aos and /tmp/maos-$USER at load time.  The
 * Makefile compiles that file with mymkdir renamed to this no-op so loading
 * the reference library creates no folders. */
void maosref_skip_mkdir(const char *format, ...) { (void)format; }
