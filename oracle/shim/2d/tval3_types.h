/* Oracle shim (test infrastructure only): the reference's missing
 * tval3_types.h = the interface's option/info/exception types.  <iostream>
 * is pulled in because 3d/tval3_cpu_3d.cpp:1228 writes to cout without
 * including it. */
#ifndef ORACLE_SHIM_TVAL3_TYPES_H_
#define ORACLE_SHIM_TVAL3_TYPES_H_
#include <iostream>
#include <cstring>
#include <cstdio>
#include "tval3/tval3_types.h"
#endif
