/*
 * vikalp_mps.h -- C entry points of the MPS ingest path (libvikalp.so, the
 * C++ host layer). A file read with vikalp::MpsReader (the reference's format
 * rules, include/vikalp/io/MpsReader.hpp) becomes a vk_problem that
 * vk_pdhg_create / vk_batch_solve accept directly. Replaces, for callers of
 * this library, the reference's MpsReader::read(path, Model&)
 * (src/io/MpsReader.cpp:10-559).
 */
#ifndef VIKALP_MPS_H
#define VIKALP_MPS_H

#include "vikalp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vk_mps vk_mps;

/* Reads `path`. Returns VK_OK, or VK_ERR_INVALID when the file has problems
 * (vk_mps_error_count / vk_mps_error list them with their lines, 0 for
 * problems found after reading) or the model it describes fails the model
 * checks (no listed errors then, as MpsReader::errors() in the reference;
 * vk_pdhg_create reports the check's message). *out is set in both cases;
 * free it with vk_mps_free. */
int vk_mps_read(const char *path, vk_mps **out);
/* Fills *problem with pointers into the model the handle owns (valid until
 * vk_mps_free) and the sizes; no quadratic objective. */
int vk_mps_problem(const vk_mps *h, vk_problem *problem, int64_t *m, int64_t *n, int64_t *nnz);
const char *vk_mps_name(const vk_mps *h);
int32_t vk_mps_binary_count(const vk_mps *h); /* variables declared BV */
int32_t vk_mps_error_count(const vk_mps *h);
const char *vk_mps_error(const vk_mps *h, int32_t index, int64_t *line);
void vk_mps_free(vk_mps *h);

#ifdef __cplusplus
}
#endif
#endif /* VIKALP_MPS_H */
