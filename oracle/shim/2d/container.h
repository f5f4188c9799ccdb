/* Oracle shim (test infrastructure only): the reference's missing container.h
 * for its 2d/ build = the interface's containers + the 2D ray geometry. */
#ifndef ORACLE_SHIM_CONTAINER_H_
#define ORACLE_SHIM_CONTAINER_H_
#include <algorithm>
#include "tval3/container.h"
#include "tval3/geometry_2d.h"
#endif
