/* Oracle shim (test infrastructure only): the reference's missing
 * timestamp.h.  get_timestamp() itself is defined by the reference's own
 * utility.h (2d/utility.h:43-51), so this header only supplies <sys/time.h>. */
#ifndef ORACLE_SHIM_TIMESTAMP_H_
#define ORACLE_SHIM_TIMESTAMP_H_
#include <sys/time.h>
#endif
