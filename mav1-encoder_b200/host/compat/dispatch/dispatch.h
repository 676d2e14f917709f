/* The reference's tile writer includes Apple's libdispatch header, which
 * Linux does not have. host/writer.c defines the one macro that file uses
 * (dispatch_apply) before including it and runs the tile columns on the host
 * driver's own thread pool, so this header is intentionally empty. */
#ifndef MH_COMPAT_DISPATCH_H
#define MH_COMPAT_DISPATCH_H
#endif
