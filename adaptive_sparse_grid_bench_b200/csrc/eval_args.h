/*
 * Arguments of the evaluation kernels and the per-dimension launchers
 * (instantiated in eval_d*.cu so that the kernels compile in parallel).
 */
#ifndef SG_EVAL_ARGS_H
#define SG_EVAL_ARGS_H

#include <stdint.h>

#include <vector_types.h>

#include "sg_kernels.h"

typedef sg_eval_args EvalArgs;

/* Unrolled-block thresholds of the wide blocking preset: 3-D blocks of
 * budget <= SG_EVAL_MAX_RF, leaf subtrees of the last prefix dim of budget
 * <= SG_EVAL_MAX_LEAF_P1 / _P2 (one / two points per thread), of the last
 * two prefix dims of budget <= SG_EVAL_MAX_LEAF2.  The medium preset unrolls
 * 3-D blocks of budget <= 5 and leaf subtrees of budget <= 3. */
#define SG_EVAL_MAX_RF 6
#define SG_EVAL_MAX_LEAF_P1 5
#define SG_EVAL_MAX_LEAF_P2 4
#define SG_EVAL_MAX_LEAF2 3

template <int D>
int eval_launch(const EvalArgs &A, int ppt, int blocking, void *stream);

/* Sets the kernels' dynamic shared memory limit on the current device. */
template <int D>
int eval_setup();

/* Points per CTA of the evaluation kernels for `ppt` points per thread. */
#define SG_EVAL_CTA_POINTS(ppt) (256 * (ppt))

/* Batched form: items[b] = (grid index into `grids` | part << 29, first
 * point) for CTA b;
 * every grid of the launch has dimension D. */
template <int D>
int eval_batch_launch(const EvalArgs *grids, const int2 *items, int nitems, int ppt, int blocking, void *stream);

#endif
