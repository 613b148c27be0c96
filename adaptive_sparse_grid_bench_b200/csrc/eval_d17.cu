/* Evaluation kernels for d = 17 and 18 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<17>(const EvalArgs &, int, void *);
template int eval_batch_launch<17>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<18>(const EvalArgs &, int, void *);
template int eval_batch_launch<18>(const EvalArgs *, const int2 *, int, int, void *);
