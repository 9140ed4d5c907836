/* The reference's sources.c compiled inside this harness unit for its
 * psystem_weight_srcs() and advance_cursor() (sources.c:55-78), the
 * per-tick source weights of emit_rays(). Test infrastructure only. */
#include "sources.c"
