/* Stand-in for <sys/sysctl.h>, which glibc >= 2.32 no longer ships.
 * The reference includes it only to print the host name and OS strings in the
 * header of its output file; this stub makes those calls report nothing. It is
 * used only when compiling the reference sources into the oracle build
 * (oracle/Makefile) and is never part of the product. */
#ifndef ORACLE_SHIM_SYS_SYSCTL_H
#define ORACLE_SHIM_SYS_SYSCTL_H
#include <stddef.h>
#define CTL_KERN 1
#define KERN_OSTYPE 1
#define KERN_OSRELEASE 2
#define KERN_VERSION 4
#define KERN_NODENAME 10
static inline int sysctl(int *name, int nlen, void *oldval, size_t *oldlenp,
                         void *newval, size_t newlen)
{
  (void)name; (void)nlen; (void)newval; (void)newlen;
  if (oldval && oldlenp && *oldlenp > 0) ((char *)oldval)[0] = '\0';
  return 0;
}
#endif
