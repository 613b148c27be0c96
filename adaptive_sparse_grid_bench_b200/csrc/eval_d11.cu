/* Evaluation kernels for d = 11 and 12 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<11>(const EvalArgs &, int, void *);
template int eval_batch_launch<11>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<12>(const EvalArgs &, int, void *);
template int eval_batch_launch<12>(const EvalArgs *, const int2 *, int, int, void *);
