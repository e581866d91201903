/* b200io: Matrix Market I/O of block-sparse Newton systems (host side, C ABI,
 * exported by libb200scene.so).
 *
 * The format is the one libuipc's debug dump writes and reads
 * (src/backends/cuda/utils/matrix_market.h:35-116 export_matrix_market,
 * :126-158 export_vector_market, :247-366 import_matrix_market, :376-450
 * import_vector_market; dump call site
 * src/backends/cuda/linear_system/global_linear_system.cu:34-70, scene setting
 * extras/debug/dump_linear_system):
 *   matrix: "%MatrixMarket matrix coordinate real general" (one '%': the
 *           reference prints its banner through a printf-style format, which
 *           turns "%%" into "%"), comment lines,
 *           "<rows> <cols> <entries>" in scalars, then for every stored 3x3
 *           block (in storage order) its 9 entries, block row by block row,
 *           zeros included: "<i> <j> <value %.17g>", indices 1-based by default;
 *   vector: "%MatrixMarket matrix array real general", comment lines,
 *           "<n> 1", then one "%.17g" value per line.
 * Import skips entries outside the stated size, groups the rest into 3x3
 * blocks ordered by (block row, block column) (an entry given twice keeps the
 * later value; block rows = ceil(rows / 3)); a vector file must state one
 * column and hold exactly <n> values.
 *
 * Block values here are 9 doubles in column-major order (B(p, q) at
 * [q * 3 + p]), the layout of the triplets b2s_assemble takes. All functions
 * return 0 on success and a negative code on failure (-1 I/O, -2 format,
 * -3 argument). */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

int b2io_write_block_matrix(const char* path, int32_t n_block_rows, int64_t n_blocks, const int32_t* rows,
                            const int32_t* cols, const double* vals, int one_based);
int b2io_write_vector(const char* path, int64_t n, const double* x);

/* reading a matrix: parse once into a handle, then copy the blocks out */
typedef struct b2io_matrix b2io_matrix;
int  b2io_read_block_matrix(const char* path, int one_based, b2io_matrix** out);
int  b2io_matrix_size(const b2io_matrix* m, int32_t* n_block_rows, int64_t* n_blocks, int64_t* n_entries);
int  b2io_matrix_copy(const b2io_matrix* m, int32_t* rows, int32_t* cols, double* vals);
void b2io_matrix_free(b2io_matrix* m);

/* reading a vector: with x == NULL only *n is set */
int b2io_read_vector(const char* path, int64_t capacity, double* x, int64_t* n);

#ifdef __cplusplus
}
#endif
