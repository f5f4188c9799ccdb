/*
 * Ray geometry of the 2D TVAL3 interface (one fan of straight rays between
 * integer pixel positions, traced with Bresenham's algorithm).
 *
 * The reference's definition is in its missing "container.h"; the fields are
 * those read by 2d/mat_mult.h:135-181 and 2d/tval3_cpu_2d.cpp:748:
 *   ray r = emitter*num_receivers + receiver; traced when use_path[r] != 0;
 *   the image index of pixel (x, y) is x + y*ld; every hit adds
 *   scale_factor * pixel to the ray (forward) or ray to the pixel (adjoint).
 * The measurement vector is uncompacted: b.len == num_emitters*num_receivers,
 * entries of untraced rays are rows of zeros.
 *
 * Only one of geometry_2d.h / geometry_3d.h may be included in a translation
 * unit: like the reference, which builds 2d/ and 3d/ as separate libraries,
 * both define a struct named geometry.
 */
#ifndef TVAL3_GEOMETRY_2D_H_
#define TVAL3_GEOMETRY_2D_H_
#ifdef TVAL3_GEOMETRY_3D_H_
#error "geometry_2d.h and geometry_3d.h define the same struct; include only one"
#endif

struct geometry {
	int num_emitters;
	int num_receivers;
	const int *use_path;    /* [num_emitters*num_receivers], nonzero = traced */
	const int *x_emitters;  /* [num_emitters] pixel x */
	const int *y_emitters;  /* [num_emitters] pixel y */
	const int *x_receivers; /* [num_receivers] pixel x */
	const int *y_receivers; /* [num_receivers] pixel y */
	int ld;                 /* row stride of the image (its dim_x) */
	float scale_factor;     /* weight of one pixel hit */
};

#endif /* TVAL3_GEOMETRY_2D_H_ */
