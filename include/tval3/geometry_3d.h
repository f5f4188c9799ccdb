/*
 * Ray geometry of the 3D TVAL3 interface.
 *
 * The reference's definition is in its missing "container.h"; the fields are
 * those read by 3d/mat_mult.h:164-359 and 3d/tval3_cpu_3d.cpp:1153:
 *   for each measurement position mp < numMPs, emitter e and receiver r:
 *   the pair is traced when use_path[e*num_receivers + r] != 0, and its ray
 *   index is mp*numPaths + use_path[e*num_receivers + r] - 1 (use_path holds a
 *   1-based compact index); coordinates are per measurement position,
 *   x_emitters[mp][e] etc.; voxel (x, y, z) has index x + y*rv_x + z*rv_x*rv_y.
 *   b.len == numPaths*numMPs.
 *
 * Only one of geometry_2d.h / geometry_3d.h may be included in a translation
 * unit (both define struct geometry, as the reference's 2d/ and 3d/ builds do).
 */
#ifndef TVAL3_GEOMETRY_3D_H_
#define TVAL3_GEOMETRY_3D_H_
#ifdef TVAL3_GEOMETRY_2D_H_
#error "geometry_2d.h and geometry_3d.h define the same struct; include only one"
#endif

struct geometry {
	int numMPs;         /* measurement positions */
	int numPaths;       /* compact rays per measurement position */
	int num_emitters;
	int num_receivers;
	const int *use_path;            /* [E*R]: 0 = unused, k>0 = ray k-1 */
	int *const *x_emitters;         /* [numMPs][E] voxel x */
	int *const *y_emitters;
	int *const *z_emitters;
	int *const *x_receivers;        /* [numMPs][R] voxel x */
	int *const *y_receivers;
	int *const *z_receivers;
	int rv_x, rv_y, rv_z;           /* volume extent */
	float scale_factor;             /* weight of one voxel hit */
};

#endif /* TVAL3_GEOMETRY_3D_H_ */
