/* Oracle shim (test infrastructure only): the reference's missing profile.h.
 * 3d/tval3_cpu_3d.cpp:1337-1349 and 3d/blas_wrap.h read
 * profile_info[k].{valid,name,time,runs} for k < 100 and call get_timestamp()
 * (defined later by the reference's utility.h, hence the forward declaration). */
#ifndef ORACLE_SHIM_PROFILE_H_
#define ORACLE_SHIM_PROFILE_H_
struct oracle_profile_slot {
	bool valid;
	char name[512];
	double time;
	int runs;
};
static oracle_profile_slot profile_info[100];
inline double get_timestamp();
#endif
