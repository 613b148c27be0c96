/* Evaluation kernels for d = 4 (see eval_impl.cuh); one dimension per file
 * so the instantiations compile in parallel. */
#include "eval_impl.cuh"

template int eval_launch<4>(const EvalArgs &, int, int, void *);
template int eval_setup<4>();
template int eval_batch_launch<4>(const EvalArgs *, const int2 *, int, int, int, void *);
