/* Evaluation kernels for d = 9 and 10 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<9>(const EvalArgs &, int, void *);
template int eval_batch_launch<9>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<10>(const EvalArgs &, int, void *);
template int eval_batch_launch<10>(const EvalArgs *, const int2 *, int, int, void *);
