/*
 * gb_oracle.h -- CPU oracle for the groupby engine (test infrastructure only).
 * Semantics and citations: see the header comment of gb_oracle.c.
 */
#ifndef GB_ORACLE_H
#define GB_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* A host column: libcudf type id, rows, element data, optional LSB-first
 * 32-bit validity words, and a row offset into data and mask. */
typedef struct {
  int32_t type_id;
  int64_t size;
  const void* data;
  const uint32_t* mask;
  int64_t offset;
} orc_column;

/* One aggregation request: a value column and the libcudf aggregation kinds
 * (cudf::aggregation::Kind numbering) to compute on it; ddof may be NULL. */
typedef struct {
  orc_column values;
  int32_t num_aggs;
  const int32_t* kinds;
  const int32_t* ddof;
} orc_request;

typedef struct orc_handle orc_handle;

int orc_valid_agg(int type_id, int kind);
int orc_groupby(const orc_column* keys, int nkeys, int include_null_keys,
                const orc_request* reqs, int nreq, int nthreads, orc_handle** out);
int64_t orc_num_groups(const orc_handle* h);
void orc_group_rows(const orc_handle* h, int64_t* out);
int orc_result(const orc_handle* h, int r, int j, void* out, uint8_t* valid, double* tol);
void orc_free(orc_handle* h);

#ifdef __cplusplus
}
#endif
#endif
