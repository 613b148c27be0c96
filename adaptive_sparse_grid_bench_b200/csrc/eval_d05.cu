/* Evaluation kernels for d = 5 and 6 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<5>(const EvalArgs &, int, void *);
template int eval_batch_launch<5>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<6>(const EvalArgs &, int, void *);
template int eval_batch_launch<6>(const EvalArgs *, const int2 *, int, int, void *);
