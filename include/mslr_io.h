/*
 * mslr_io.h — C ABI of libmslrio.so, the MAT v7.3 (HDF5) reader and writer
 * for run_recon's input and output files.  Host code only (no GPU needed).
 *
 * Replaces, for the files run_recon touches:
 *   - h5read(fn_ksp, "ksp_epi_zf")        scripts/reconstruct.jl:95  (HDF5.jl)
 *   - matread(fn_smaps)["smaps"]          scripts/reconstruct.jl:88  (MAT.jl)
 *   - matwrite(fn_out, Dict(...); compress=true)
 *                                         scripts/reconstruct.jl:242-260 (MAT.jl)
 *
 * A MAT v7.3 file is an HDF5 file behind a 512-byte MATLAB header (the HDF5
 * "user block").  The reader handles what MATLAB and libhdf5 write for such
 * files: superblocks 0-3; object headers 1 and 2 with continuation blocks;
 * symbol-table groups, compact link messages and dense link storage (a
 * fractal heap with a one- or two-level name index); fixed-point, IEEE float,
 * complex (a compound of two floats named real/imag, r/i or re/im), string
 * and object-reference datatypes; contiguous, compact and chunked layouts
 * (layout messages 1-4; chunk indexes: version-1 B-tree, single chunk,
 * implicit, fixed array); the deflate, shuffle and Fletcher-32 filters.
 * Not handled (reported as MSLRIO_ERR_UNSUPPORTED): fractal heaps with
 * filters, huge objects or nested indirect blocks, deeper name indexes,
 * extensible-array and version-2 B-tree chunk indexes,
 * big-endian data, variable-length types, external and virtual storage.
 *
 * The writer produces the structure MATLAB writes for `save -v7.3`:
 * superblock 0 at offset 512 behind the MATLAB header, version-1 object
 * headers, symbol-table groups, layout message 3 (contiguous, or chunked with
 * a version-1 B-tree chunk index and the deflate filter), and the
 * MATLAB_class / MATLAB_int_decode / MATLAB_empty attributes.
 *
 * Conventions:
 *   - dims are HDF5's, slowest first: a Julia / MATLAB array of size
 *     (d1, ..., dn) is stored with dims (dn, ..., d1) and the same bytes, so
 *     the data buffers here are C-order arrays with the HDF5 dims;
 *   - complex elements are interleaved (re, im) pairs;
 *   - objects are named by path ("/ksp_epi_zf", "/#refs#/a") or by their
 *     object-header address (what an object reference holds);
 *   - every call returns an int status (MSLRIO_OK == 0) and never aborts;
 *     mslrio_last_error() gives the calling thread's last failure message;
 *   - one file handle may be read from several host threads at once (the
 *     handle is immutable after mslrio_open); a writer handle may not.
 */
#ifndef MSLR_IO_H
#define MSLR_IO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSLRIO_OK 0
#define MSLRIO_ERR_ARG 1          /* bad argument (size, name, buffer) */
#define MSLRIO_ERR_IO 2           /* open / read / write / mmap failed */
#define MSLRIO_ERR_FORMAT 3       /* the file is not HDF5 or is damaged */
#define MSLRIO_ERR_UNSUPPORTED 4  /* HDF5 feature outside the supported set */
#define MSLRIO_ERR_NOTFOUND 5     /* no object of that name */

/* Element types (mslrio_info.dtype, mslrio_write `dtype`). */
#define MSLRIO_I8 1
#define MSLRIO_U8 2
#define MSLRIO_I16 3
#define MSLRIO_U16 4
#define MSLRIO_I32 5
#define MSLRIO_U32 6
#define MSLRIO_I64 7
#define MSLRIO_U64 8
#define MSLRIO_F32 9
#define MSLRIO_F64 10
#define MSLRIO_C64 11             /* compound {real f32, imag f32} */
#define MSLRIO_C128 12            /* compound {real f64, imag f64} */
#define MSLRIO_REF 13             /* object reference: 8-byte object-header address */
#define MSLRIO_STR 14             /* fixed-length string, elem_size bytes */
#define MSLRIO_GROUP 100          /* the object is a group, not a dataset */

#define MSLRIO_MAX_RANK 32

typedef struct mslrio_file mslrio_file;
typedef struct mslrio_writer mslrio_writer;

typedef struct {
    uint64_t addr;                     /* object-header address (file-relative) */
    int32_t dtype;                     /* MSLRIO_* element type or MSLRIO_GROUP */
    int32_t elem_size;                 /* bytes per element */
    int32_t rank;                      /* 0 = scalar dataspace */
    int32_t layout;                    /* 0 compact, 1 contiguous, 2 chunked */
    int64_t dims[MSLRIO_MAX_RANK];     /* slowest first */
    int64_t chunk[MSLRIO_MAX_RANK];    /* chunk dims when chunked */
    int32_t n_filters;                 /* filters in the pipeline */
    int32_t matlab_int_decode;         /* MATLAB_int_decode attribute, -1 if absent */
    int32_t matlab_empty;              /* MATLAB_empty attribute (0 if absent) */
    char matlab_class[32];             /* MATLAB_class attribute, "" if absent */
} mslrio_info;

/* Open an HDF5 / MAT v7.3 file for reading (memory-mapped).  Replaces the
 * file handling of h5read / matread (scripts/reconstruct.jl:88,95). */
int mslrio_open(const char* path, mslrio_file** out);
int mslrio_close(mslrio_file* f);

/* Byte offset of the HDF5 superblock (512 for MAT v7.3 files). */
int mslrio_userblock(const mslrio_file* f, uint64_t* bytes);

/* Members of a group (path "/" for the root): count, then the i-th name. */
int mslrio_group_count(mslrio_file* f, const char* group, int32_t* n);
int mslrio_group_name(mslrio_file* f, const char* group, int32_t i, char* buf, size_t cap);

/* Object-header address of a path; then its description. */
int mslrio_lookup(mslrio_file* f, const char* path, uint64_t* addr);
int mslrio_info_at(mslrio_file* f, uint64_t addr, mslrio_info* info);

/* Read a whole dataset into dst (C order, HDF5 dims, elem_size bytes per
 * element; dst_bytes must equal the product of dims × elem_size).  Chunks
 * are decoded on `nthreads` host threads (<= 0: all cores).  Chunks that
 * the file never wrote read as zeros (the default fill value). */
int mslrio_read_at(mslrio_file* f, uint64_t addr, void* dst, size_t dst_bytes, int32_t nthreads);

/* Create a file for writing.  matlab_header != 0 writes the 512-byte MATLAB
 * v7.3 header ("MATLAB 7.3 MAT-file ...") as the HDF5 user block. */
int mslrio_create(const char* path, int32_t matlab_header, mslrio_writer** out);

/* Write one dataset.  `name` is "var" (root group) or "grp/var" (one level
 * of subgroup, created on first use, e.g. MATLAB's "#refs#" group that holds
 * cell elements).  dims are slowest first; data is C order.  matlab_class ""
 * writes no MATLAB_class attribute; matlab_int_decode < 0 writes none;
 * matlab_empty != 0 writes MATLAB_empty = 1.  deflate_level 0 stores the
 * data contiguously; 1-9 stores it in chunks of about chunk_bytes (<= 0:
 * 4 MiB) compressed with zlib at that level on `nthreads` threads (a chunk
 * that does not shrink is stored raw, its filter-mask bit set).  The new
 * object's header address is returned in *addr (for object references). */
int mslrio_write(mslrio_writer* w, const char* name, int32_t dtype, int32_t rank, const int64_t* dims,
                 const void* data, const char* matlab_class, int32_t matlab_int_decode,
                 int32_t matlab_empty, int32_t deflate_level, int64_t chunk_bytes, int32_t nthreads,
                 uint64_t* addr);

/* Write the groups and the superblock and close the file; the handle is
 * freed either way.  mslrio_abort closes and deletes the partial file. */
int mslrio_finish(mslrio_writer* w);
int mslrio_abort(mslrio_writer* w);

const char* mslrio_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MSLR_IO_H */
