/* Oracle build only (test infrastructure). The reference's tile writer
 * includes <dispatch/dispatch.h> (Apple libdispatch), which does not exist on
 * Linux. oracle/ref_tile.c defines the one macro that file uses before
 * including it, so this header is intentionally empty. */
#ifndef ORACLE_COMPAT_DISPATCH_H
#define ORACLE_COMPAT_DISPATCH_H
#endif
