// Instantiations of the fused draw kernel: double, N in {192, 256, 384, 512, 768, 1024}.
// Split from the other sizes so the heavily unrolled kernels compile in parallel.
#include "gsb_draw.cuh"

namespace gsb {

int fused_launch_f64_large(int N, const DrawArgs& args, size_t work_bytes, cudaStream_t stream, bool* handled)
{
    *handled = true;
    switch (N) {
      case 192: return launch_fused<double, 192>(args, work_bytes, stream);
      case 256: return launch_fused<double, 256>(args, work_bytes, stream);
      case 384: return launch_fused<double, 384>(args, work_bytes, stream);
      case 512: return launch_fused<double, 512>(args, work_bytes, stream);
      case 768: return launch_fused<double, 768>(args, work_bytes, stream);
      case 1024: return launch_fused<double, 1024>(args, work_bytes, stream);
    }
    *handled = false;
    return GSB_OK;
}

bool fused_workspace_f64_large(int N, int n_stamps, size_t* bytes)
{
    switch (N) {
      case 192: *bytes = workspace_bytes_for<double, 192>(n_stamps); return true;
      case 256: *bytes = workspace_bytes_for<double, 256>(n_stamps); return true;
      case 384: *bytes = workspace_bytes_for<double, 384>(n_stamps); return true;
      case 512: *bytes = workspace_bytes_for<double, 512>(n_stamps); return true;
      case 768: *bytes = workspace_bytes_for<double, 768>(n_stamps); return true;
      case 1024: *bytes = workspace_bytes_for<double, 1024>(n_stamps); return true;
    }
    return false;
}

}  // namespace gsb
