// Instantiations of the fused particle kernel for shape order 3.
#include "pxr_cell_kernel.cuh"

namespace pxrt {
template <typename R, int ORDER, int T, int D, int MODE>
int launch_step(const Job* jobs, const int2* work, int nwork, const int* nwork_dev, int* ctr,
                int threads, int ctas, size_t smem, cudaStream_t s) {
  auto kern = k_tile_step<R, ORDER, T, D, MODE>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return PXRB_EUNSUPPORTED;
  if (cudaMemsetAsync(ctr, 0, sizeof(int), s) != cudaSuccess) return PXRB_ELAUNCH;
  kern<<<ctas, threads, smem, s>>>(jobs, work, nwork, nwork_dev, ctr);
  PXRB_CHECK_LAUNCH();
  return PXRB_OK;
}

template <typename R, int ORDER>
int launch_shape(int tile, int drift, int mode, const Job* jobs, const int2* work, int nwork,
                 const int* nwork_dev, int* ctr, int threads, int ctas, size_t smem,
                 cudaStream_t s) {
#define PXRB_TD(T_, D_, M_)                                                                  \
  if (tile == T_ && drift == D_ && mode == M_)                                              \
    return launch_step<R, ORDER, T_, D_, M_>(jobs, work, nwork, nwork_dev, ctr, threads,    \
                                             ctas, smem, s);
  if (mode == 4) {       // cell-grouped kernel (FP32, int32 fixed point)
    if (sizeof(R) != 4) return PXRB_EUNSUPPORTED;
    if (tile == 8 && drift == 1)
      return launch_cell<ORDER, 8, 1>(jobs, work, nwork, nwork_dev, ctr, threads, ctas, smem, s);
    return PXRB_EUNSUPPORTED;
  }
  if (sizeof(R) == 8) {
    PXRB_TD(8, 1, 3)
    PXRB_TD(8, 0, 3)
    PXRB_TD(4, 1, 3)
    PXRB_TD(4, 0, 3)
  } else {
    PXRB_TD(8, 1, 2)
    PXRB_TD(8, 1, 1)
    PXRB_TD(8, 1, 0)
    PXRB_TD(8, 0, 2)
    PXRB_TD(8, 2, 2)
    PXRB_TD(8, 2, 1)
    PXRB_TD(4, 1, 2)
    PXRB_TD(4, 1, 1)
    PXRB_TD(4, 0, 2)
  }
#undef PXRB_TD
  return PXRB_EUNSUPPORTED;
}


int launch_order3(int prec, int tile, int drift, int mode, const pxrb_tiled_job* jobs,
                  const int2* work, int nwork, const int* nwork_dev, int* ctr, int threads,
                  int ctas, size_t smem, cudaStream_t s) {
  if (prec == 0)
    return launch_shape<float, 3>(tile, drift, mode, jobs, work, nwork, nwork_dev, ctr,
                                    threads, ctas, smem, s);
  return launch_shape<double, 3>(tile, drift, mode, jobs, work, nwork, nwork_dev, ctr,
                                   threads, ctas, smem, s);
}
}  // namespace pxrt

extern "C" int32_t pxrb_tiled_max_threads(int32_t acc) {
  return acc == 4 ? pxrt::CG_THREADS : acc == 3 ? pxrt::MAX_THREADS_FP64 : pxrt::MAX_THREADS;
}
