/* Force-included into every reference translation unit by oracle/ref/Makefile.
 * glibc >= 2.32 no longer declares sys_siglist; the reference prints signal
 * names through it, so map it onto a table filled from strsignal(). */
#ifndef MAOSREF_SHIM_COMPAT_H
#define MAOSREF_SHIM_COMPAT_H
extern const char *maosref_siglist[65];
#define sys_siglist maosref_siglist
#endif
