/* fastwarp_transform_io.h -- the transform files a registration writes, in ITK's formats.
 *
 * Replaces the reference's output writers (crates/fastwarp-reg/src/stages.rs:405-560,
 * write_stage_outputs with OutputLayout::Composite): Composite.h5 and InverseComposite.h5
 * (transform/itk_h5.rs:108-200, format_h5 / write_h5_to, over the HDF5 subset writer of
 * transform/hdf5.rs:1127-1400) and 0GenericAffine.mat (transform/itk_mat.rs:134-181,
 * format_mat / write_mat_file). The bytes are the reference's: superblock version 2,
 * version-2 object headers without timestamps, compact groups, contiguous f64 datasets (field
 * displacements widened from float32), variable-length strings in one global heap.
 *
 * Host code only; no device is needed. Every function returns 0 or a non-zero status with the
 * message in fw_last_error() (include/fastwarp_cuda.h).
 */
#ifndef FASTWARP_TRANSFORM_IO_H
#define FASTWARP_TRANSFORM_IO_H

#include <stddef.h>
#include <stdint.h>

#include "fastwarp_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FW_ELEM_AFFINE 0
#define FW_ELEM_FIELD 1

/* One transform of a chain (TransformElem, transform/composite.rs). An affine maps
 * x -> M (x - c) + t + c (ITK AffineTransform: parameters M row-major then t, fixed parameters c).
 * A displacement field lives on `grid` with `field` its displacements, AoS float32 (x, y, z per
 * voxel, x fastest: the reference's DisplacementField::data layout). */
typedef struct fw_transform_elem {
    int32_t kind; /* FW_ELEM_AFFINE or FW_ELEM_FIELD */
    double matrix[9];
    double translation[3];
    double center[3];
    fw_grid grid;
    const float* field;
} fw_transform_elem;

/* HDF5's metadata checksum: Jenkins' lookup3 hashlittle with initval 0 (transform/hdf5.rs:48-113). */
uint32_t fw_lookup3(const uint8_t* data, size_t len);

/* format_h5 (transform/itk_h5.rs:108-190): the bytes of an ITK composite transform file of the
 * chain in queue order (TransformGroup/0 the composite, /1.. the elements). `os_name` and
 * `os_version` are the OSName / OSVersion strings (the reference writes Rust's
 * std::env::consts::OS and ARCH; NULL gives "linux" and "x86_64"). With `out` NULL or `cap` too
 * small nothing is written and *len receives the size needed. An empty chain is an error. */
int fw_format_itk_h5(const fw_transform_elem* chain, int32_t n, const char* os_name,
                     const char* os_version, uint8_t* out, size_t cap, size_t* len);
/* write_h5_file: the same bytes streamed to `path` (through a temporary file renamed on success,
 * as fs_write::write_complete does). */
int fw_write_itk_h5(const char* path, const fw_transform_elem* chain, int32_t n);

/* format_mat (transform/itk_mat.rs:148-165): every element an affine; 193 bytes per affine. */
int fw_format_itk_mat(const fw_transform_elem* chain, int32_t n, uint8_t* out, size_t cap,
                      size_t* len);
int fw_write_itk_mat(const char* path, const fw_transform_elem* chain, int32_t n);

#ifdef __cplusplus
}
#endif

#endif
