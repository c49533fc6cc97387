// Instantiations of the fused adjoint kernel: double, N = 2^a or 3*2^a in 32..1024.
#include "gsb_adjoint.cuh"

namespace gsb {

int adjoint_launch_f64(int N, const AdjArgs& args, size_t work_bytes, cudaStream_t stream, bool* handled)
{
    *handled = true;
    switch (N) {
      case 32: return launch_adjoint<double, 32>(args, work_bytes, stream);
      case 48: return launch_adjoint<double, 48>(args, work_bytes, stream);
      case 64: return launch_adjoint<double, 64>(args, work_bytes, stream);
      case 96: return launch_adjoint<double, 96>(args, work_bytes, stream);
      case 128: return launch_adjoint<double, 128>(args, work_bytes, stream);
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

bool adjoint_workspace_f64(int N, int n_stamps, size_t* bytes)
{
    switch (N) {
      case 32: *bytes = adj_workspace_bytes_for<double, 32>(n_stamps); return true;
      case 48: *bytes = adj_workspace_bytes_for<double, 48>(n_stamps); return true;
      case 64: *bytes = adj_workspace_bytes_for<double, 64>(n_stamps); return true;
      case 96: *bytes = adj_workspace_bytes_for<double, 96>(n_stamps); return true;
      case 128: *bytes = adj_workspace_bytes_for<double, 128>(n_stamps); return true;
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
