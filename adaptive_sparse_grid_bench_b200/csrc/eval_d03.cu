/* Evaluation kernels for d = 3 and 4 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<3>(const EvalArgs &, int, void *);
template int eval_batch_launch<3>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<4>(const EvalArgs &, int, void *);
template int eval_batch_launch<4>(const EvalArgs *, const int2 *, int, int, void *);
