/* Evaluation kernels for d = 7 and 8 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<7>(const EvalArgs &, int, void *);
template int eval_batch_launch<7>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<8>(const EvalArgs &, int, void *);
template int eval_batch_launch<8>(const EvalArgs *, const int2 *, int, int, void *);
