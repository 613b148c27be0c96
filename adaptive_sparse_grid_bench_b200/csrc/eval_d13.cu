/* Evaluation kernels for d = 13 and 14 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<13>(const EvalArgs &, int, void *);
template int eval_batch_launch<13>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<14>(const EvalArgs &, int, void *);
template int eval_batch_launch<14>(const EvalArgs *, const int2 *, int, int, void *);
