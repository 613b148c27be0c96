/* Evaluation kernels for d = 19 and 20 (see eval_impl.cuh). */
#include "eval_impl.cuh"

template int eval_launch<19>(const EvalArgs &, int, void *);
template int eval_batch_launch<19>(const EvalArgs *, const int2 *, int, int, void *);
template int eval_launch<20>(const EvalArgs &, int, void *);
template int eval_batch_launch<20>(const EvalArgs *, const int2 *, int, int, void *);
