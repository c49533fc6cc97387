// Instantiations of the fused adjoint kernel: double, N in {192, 256, 384, 512, 768, 1024}.
// Split by size group so the unrolled kernels compile in parallel.
#include "gsb_adjoint.cuh"

namespace gsb {

int adjoint_launch_f64_large(int N, const AdjArgs& args, size_t work_bytes, cudaStream_t stream, bool* handled)
{
    *handled = true;
    switch (N) {
      case 192: return launch_adjoint<double, 192>(args, work_bytes, stream);
      case 256: return launch_adjoint<double, 256>(args, work_bytes, stream);
      case 384: return launch_adjoint<double, 384>(args, work_bytes, stream);
      case 512: return launch_adjoint<double, 512>(args, work_bytes, stream);
      case 768: return launch_adjoint<double, 768>(args, work_bytes, stream);
      case 1024: return launch_adjoint<double, 1024>(args, work_bytes, stream);
    }
    *handled = false;
    return GSB_OK;
}

bool adjoint_workspace_f64_large(int N, int n_stamps, size_t* bytes)
{
    switch (N) {
      case 192: *bytes = adj_workspace_bytes_for<double, 192>(n_stamps); return true;
      case 256: *bytes = adj_workspace_bytes_for<double, 256>(n_stamps); return true;
      case 384: *bytes = adj_workspace_bytes_for<double, 384>(n_stamps); return true;
      case 512: *bytes = adj_workspace_bytes_for<double, 512>(n_stamps); return true;
      case 768: *bytes = adj_workspace_bytes_for<double, 768>(n_stamps); return true;
      case 1024: *bytes = adj_workspace_bytes_for<double, 1024>(n_stamps); return true;
    }
    return false;
}

}  // namespace gsb
