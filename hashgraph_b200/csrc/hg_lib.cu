// hg_lib.cu -- single translation unit of libhashgraph_b200.so.  The kernels
// share one __device__ error word, so the sources are compiled together
// rather than with relocatable device code.
#include "hg_build.cu"
#include "hg_probe.cu"
#include "hg_gen.cu"
#include "hg_api.cu"
#include "hg_noalloc.cu"
#include "hg_batch.cu"
#include "hg_io.cu"
#include "hg_server.cu"
#include "hg_shard.cu"
