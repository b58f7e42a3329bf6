// temporary: 3D, batch and serving paths are added next
#include "engine.cuh"
namespace orf {
}
extern "C" {
int32_t orf_serve_open(orf_ctx*, const orf_serve_cfg*, orf_server**) { return ORF_EINVAL; }
int32_t orf_serve_submit2d(orf_server*, const orf_sim2d*, orf_out2d*, int64_t*) { return ORF_EINVAL; }
int32_t orf_serve_submit3d(orf_server*, const orf_sim3d*, orf_out3d*, int64_t*) { return ORF_EINVAL; }
int32_t orf_serve_step(orf_server*) { return ORF_EINVAL; }
int32_t orf_serve_poll(orf_server*, int64_t, orf_serve_job_info*) { return ORF_EINVAL; }
int32_t orf_serve_pending(orf_server*, int32_t*, int32_t*) { return ORF_EINVAL; }
double orf_serve_clock(orf_server*) { return 0; }
int32_t orf_serve_close(orf_server*) { return ORF_EINVAL; }
}
