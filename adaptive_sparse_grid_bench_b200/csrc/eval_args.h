/*
 * Arguments of the evaluation kernels and the per-dimension launchers
 * (instantiated in eval_d*.cu so that the kernels compile in parallel).
 */
#ifndef SG_EVAL_ARGS_H
#define SG_EVAL_ARGS_H

#include <stdint.h>

#include "sg_kernels.h"

struct EvalArgs {
    const float *__restrict__ alpha;          /* block layout                 */
    const float *__restrict__ coords;
    const int32_t *__restrict__ perm;
    float *__restrict__ out;
    int64_t num_evals;
    int nm1;                                  /* n - 1                        */
    int regular;                              /* innermost dims unrestricted  */
    int lim[SG_MAX_DIMS];
    uint32_t blk3[SG_MAX_LEVELS];             /* block size per budget R      */
    uint32_t blk2[SG_MAX_LEVELS];             /* sub-block size per budget r  */
};

template <int D>
int eval_launch(const EvalArgs &A, int ppt, void *stream);

#endif
