/*
 * Dense and sparse containers of the TVAL3 C++ interface.
 *
 * The reference (modk/tval3-cpu) includes "container.h" but does not ship it
 * (2d/mat_mult.h:6, 3d/mat_mult.h:7).  The class layout below is inferred from
 * every use in 2d/tval3_cpu_2d.cpp and 3d/tval3_cpu_3d.cpp:
 *
 *   mat<T>          dim_x, dim_y, dim_z, len, format, data(), operator[],
 *                   ctors (len), (dim_y, dim_x), (dim_y, dim_x, dim_z), deep copy.
 *                   Storage is zero-initialised: the solver relies on it for the
 *                   multipliers delta/sigma (2d/tval3_cpu_2d.cpp:165-167) and for
 *                   the beta=1 gemm into a fresh matrix (2d/mat_mult.h:24-30).
 *                   Assignment between matrices of equal length copies the
 *                   elements only and keeps the destination's shape: the solver
 *                   assigns length-only vectors to shaped images
 *                   (U = data.Atb, 2d/tval3_cpu_2d.cpp:775; data.d = DtsAtd,
 *                   2d/tval3_cpu_2d.cpp:582) and then reads the image's dim_x /
 *                   dim_y again (2d/tval3_cpu_2d.cpp:431-433).
 *   sparse_mat<T>   dim_y (rows, m), dim_x (columns, n), nnz, format,
 *                   csr_val/ind/ptr(), csc_val/ind/ptr(); 0-based int32 indices,
 *                   ptr arrays of length rows+1 / columns+1 (the solver passes
 *                   ptr and ptr+1 as MKL's pointerB/pointerE,
 *                   2d/mat_mult.h:58-66).
 *
 * Element index convention (both 2D and 3D): i = x + y*dim_x + z*dim_x*dim_y,
 * x fastest, whatever the format flag says (2d/tval3_cpu_2d.cpp:268-293).
 *
 * This header compiles as C++98 so that the reference sources can be built
 * against it unchanged (they need -std=gnu++98).
 */
#ifndef TVAL3_CONTAINER_H_
#define TVAL3_CONTAINER_H_

#include <cstdlib>
#include <cstring>
#include <new>

enum mat_format { mat_row_major = 0, mat_col_major = 1 };

enum sparse_mat_format { sparse_mat_csr = 0, sparse_mat_csc = 1, sparse_mat_both = 2 };

template <class T>
class mat {
public:
	int dim_x;
	int dim_y;
	int dim_z;
	int len;
	mat_format format;

	explicit mat(int len_ = 0, mat_format fmt = mat_col_major)
		: dim_x(1), dim_y(len_), dim_z(1), len(len_), format(fmt), buf(0) {
		alloc();
	}
	mat(int dim_y_, int dim_x_, mat_format fmt = mat_col_major)
		: dim_x(dim_x_), dim_y(dim_y_), dim_z(1), len(dim_x_ * dim_y_),
		  format(fmt), buf(0) {
		alloc();
	}
	mat(int dim_y_, int dim_x_, int dim_z_, mat_format fmt = mat_col_major)
		: dim_x(dim_x_), dim_y(dim_y_), dim_z(dim_z_),
		  len(dim_x_ * dim_y_ * dim_z_), format(fmt), buf(0) {
		alloc();
	}
	mat(const mat &o)
		: dim_x(o.dim_x), dim_y(o.dim_y), dim_z(o.dim_z), len(o.len),
		  format(o.format), buf(0) {
		alloc();
		if (len > 0) std::memcpy(buf, o.buf, sizeof(T) * (size_t)len);
	}
	~mat() { std::free(buf); }

	mat &operator=(const mat &o) {
		if (this == &o) return *this;
		if (o.len != len) {
			/* different length: become a full copy (shape included) */
			std::free(buf);
			buf = 0;
			dim_x = o.dim_x; dim_y = o.dim_y; dim_z = o.dim_z; len = o.len;
			format = o.format;
			alloc();
		}
		if (len > 0) std::memcpy(buf, o.buf, sizeof(T) * (size_t)len);
		return *this;
	}

	T *data() { return buf; }
	const T *data() const { return buf; }
	T &operator[](int i) { return buf[i]; }
	const T &operator[](int i) const { return buf[i]; }

private:
	T *buf;
	void alloc() {
		if (len > 0) {
			buf = static_cast<T *>(std::calloc((size_t)len, sizeof(T)));
			if (!buf) throw std::bad_alloc();
		}
	}
};

template <class T>
class sparse_mat {
public:
	int dim_y;  /* rows (measurements, m) */
	int dim_x;  /* columns (pixels / voxels, n) */
	int nnz;
	sparse_mat_format format;

	sparse_mat(int dim_y_ = 0, int dim_x_ = 0, int nnz_ = 0,
	           sparse_mat_format fmt = sparse_mat_both)
		: dim_y(dim_y_), dim_x(dim_x_), nnz(nnz_), format(fmt),
		  r_val(0), r_ind(0), r_ptr(0), c_val(0), c_ind(0), c_ptr(0) {
		r_val = alloc<T>(nnz); r_ind = alloc<int>(nnz); r_ptr = alloc<int>(dim_y + 1);
		c_val = alloc<T>(nnz); c_ind = alloc<int>(nnz); c_ptr = alloc<int>(dim_x + 1);
	}
	~sparse_mat() {
		std::free(r_val); std::free(r_ind); std::free(r_ptr);
		std::free(c_val); std::free(c_ind); std::free(c_ptr);
	}

	T *csr_val() { return r_val; }
	int *csr_ind() { return r_ind; }
	int *csr_ptr() { return r_ptr; }
	T *csc_val() { return c_val; }
	int *csc_ind() { return c_ind; }
	int *csc_ptr() { return c_ptr; }
	const T *csr_val() const { return r_val; }
	const int *csr_ind() const { return r_ind; }
	const int *csr_ptr() const { return r_ptr; }
	const T *csc_val() const { return c_val; }
	const int *csc_ind() const { return c_ind; }
	const int *csc_ptr() const { return c_ptr; }

	/* Fill the CSC arrays from the CSR arrays (stable: rows ascending within
	 * each column). */
	void build_csc_from_csr() {
		for (int j = 0; j <= dim_x; j++) c_ptr[j] = 0;
		for (int k = 0; k < nnz; k++) c_ptr[r_ind[k] + 1]++;
		for (int j = 0; j < dim_x; j++) c_ptr[j + 1] += c_ptr[j];
		int *next = alloc<int>(dim_x + 1);
		for (int j = 0; j <= dim_x; j++) next[j] = c_ptr[j];
		for (int i = 0; i < dim_y; i++)
			for (int k = r_ptr[i]; k < r_ptr[i + 1]; k++) {
				int p = next[r_ind[k]]++;
				c_ind[p] = i;
				c_val[p] = r_val[k];
			}
		std::free(next);
	}

private:
	sparse_mat(const sparse_mat &);
	sparse_mat &operator=(const sparse_mat &);
	T *r_val; int *r_ind; int *r_ptr;
	T *c_val; int *c_ind; int *c_ptr;
	template <class U> static U *alloc(int count) {
		if (count <= 0) count = 1;
		U *p = static_cast<U *>(std::calloc((size_t)count, sizeof(U)));
		if (!p) throw std::bad_alloc();
		return p;
	}
};

#endif /* TVAL3_CONTAINER_H_ */
