// pending.cu — entry points whose kernels are not in this build yet.
#include "ctx.h"
using namespace rkf;
extern "C" {
rkf_status rkf_serve_start(rkf_ctx*, const rkf_march_params*) { return fail(RKF_UNSUPPORTED, "serve: not built"); }
rkf_status rkf_serve_stop(rkf_ctx*) { return RKF_OK; }
rkf_status rkf_submit(rkf_ctx*, const rkf_request*, rkf_ticket*) { return fail(RKF_UNSUPPORTED, "serve: not built"); }
rkf_status rkf_poll(rkf_ctx*, rkf_ticket, rkf_result*, uint32_t) { return fail(RKF_UNSUPPORTED, "serve: not built"); }
rkf_status rkf_cancel(rkf_ctx*, rkf_ticket) { return fail(RKF_UNSUPPORTED, "serve: not built"); }
}
