// Instantiations of the fused adjoint kernel: float, N in {32, 48, 64, 96, 128}.
// Split by size group so the unrolled kernels compile in parallel.
#include "gsb_adjoint.cuh"

namespace gsb {

int adjoint_launch_f32_small(int N, const AdjArgs& args, size_t work_bytes, cudaStream_t stream, bool* handled)
{
    *handled = true;
    switch (N) {
      case 32: return launch_adjoint<float, 32>(args, work_bytes, stream);
      case 48: return launch_adjoint<float, 48>(args, work_bytes, stream);
      case 64: return launch_adjoint<float, 64>(args, work_bytes, stream);
      case 96: return launch_adjoint<float, 96>(args, work_bytes, stream);
      case 128: return launch_adjoint<float, 128>(args, work_bytes, stream);
    }
    *handled = false;
    return GSB_OK;
}

bool adjoint_workspace_f32_small(int N, int n_stamps, size_t* bytes)
{
    switch (N) {
      case 32: *bytes = adj_workspace_bytes_for<float, 32>(n_stamps); return true;
      case 48: *bytes = adj_workspace_bytes_for<float, 48>(n_stamps); return true;
      case 64: *bytes = adj_workspace_bytes_for<float, 64>(n_stamps); return true;
      case 96: *bytes = adj_workspace_bytes_for<float, 96>(n_stamps); return true;
      case 128: *bytes = adj_workspace_bytes_for<float, 128>(n_stamps); return true;
    }
    return false;
}

}  // namespace gsb
