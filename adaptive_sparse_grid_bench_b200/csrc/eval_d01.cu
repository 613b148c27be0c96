/* Evaluation kernels for d = 1 and 2 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<1>(const EvalArgs &, int, void *);
template int eval_batch_launch<1>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<2>(const EvalArgs &, int, void *);
template int eval_batch_launch<2>(const EvalArgs *, const int2 *, int, int, void *);
