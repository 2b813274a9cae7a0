// Local-PSF overlap-add render (placeholder until the kernels land).
#include "common.cuh"

extern "C" size_t mm_local_render_workspace_size(const mm_local_desc* desc) {
  (void)desc;
  return 0;
}

extern "C" int mm_local_render(const mm_local_desc* desc, const double* source, const double* zweight, double* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  (void)desc; (void)source; (void)zweight; (void)out; (void)workspace; (void)workspace_bytes; (void)stream;
  mm::set_error("local render not built");
  return MM_ERR_UNSUPPORTED;
}
