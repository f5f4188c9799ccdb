/*
 * Oracle (test infrastructure only): the reference's own 3D Bresenham
 * projector, gemv(TransA, const geometry &, const mat<Type> &, mat<Type> &)
 * (3d/mat_mult.h:148-595), applied in double precision to a caller's vector.
 * It is compiled from the reference's mat_mult.h where it lies (oracle/Makefile)
 * and lets the tests read each ray's voxel list straight from the reference's
 * live projector: applied to one-hot voxel vectors (small volumes) or to
 * integer moment probes (full-size geometries).
 */
#include <omp.h>

#include <cstdlib>
#include <cstring>
#include <vector>

#include "container.h"
#include "tval3_types.h"
#include "mat_mult.h"

extern "C" {

/* y = A x (trans = 0: x has rv_x*rv_y*rv_z entries, y numMPs*numPaths) or
 * y = A^T x (trans = 1); coordinates flattened as in ref3d_ray
 * (xe[mp*E + e], xr[mp*R + r]). */
int ref3d_project(int trans, int numMPs, int numPaths, int E, int R, const int *use_path, int *xe, int *ye,
                  int *ze, int *xr, int *yr, int *zr, int rv_x, int rv_y, int rv_z, float scale,
                  const double *x, double *y) {
	std::vector<int *> pxe(numMPs), pye(numMPs), pze(numMPs), pxr(numMPs), pyr(numMPs), pzr(numMPs);
	for (int i = 0; i < numMPs; i++) {
		pxe[i] = xe + (size_t)i * E; pye[i] = ye + (size_t)i * E; pze[i] = ze + (size_t)i * E;
		pxr[i] = xr + (size_t)i * R; pyr[i] = yr + (size_t)i * R; pzr[i] = zr + (size_t)i * R;
	}
	geometry g;
	g.numMPs = numMPs; g.numPaths = numPaths; g.num_emitters = E; g.num_receivers = R;
	g.use_path = use_path;
	g.x_emitters = &pxe[0]; g.y_emitters = &pye[0]; g.z_emitters = &pze[0];
	g.x_receivers = &pxr[0]; g.y_receivers = &pyr[0]; g.z_receivers = &pzr[0];
	g.rv_x = rv_x; g.rv_y = rv_y; g.rv_z = rv_z; g.scale_factor = scale;
	const int nvox = rv_x * rv_y * rv_z, nray = numMPs * numPaths;
	mat<double> xv(trans ? nray : nvox), yv(trans ? nvox : nray);
	std::memcpy(xv.data(), x, sizeof(double) * (size_t)xv.len);
	gemv(trans ? CblasTrans : CblasNoTrans, g, xv, yv);
	std::memcpy(y, yv.data(), sizeof(double) * (size_t)yv.len);
	return 0;
}

}
