/* Evaluation kernels for d = 15 and 16 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<15>(const EvalArgs &, int, void *);
template int eval_batch_launch<15>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<16>(const EvalArgs &, int, void *);
template int eval_batch_launch<16>(const EvalArgs *, const int2 *, int, int, void *);
