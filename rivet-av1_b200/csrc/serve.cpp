// serve.cpp — placeholder of the serving API until the request loop lands.
#include "av1pf.h"
#include "ctx.h"

extern "C" {
int av1pf_serve_open(av1pf_ctx*, const av1pf_serve_config*, av1pf_server** out) {
  if (out) *out = nullptr;
  av1pf::set_error("serving is not built yet");
  return AV1PF_ERR_UNSUPPORTED;
}
int av1pf_serve_open_stream(av1pf_server*, const av1pf_frame_info*, int32_t*) { return AV1PF_ERR_UNSUPPORTED; }
int av1pf_serve_close_stream(av1pf_server*, int32_t) { return AV1PF_ERR_UNSUPPORTED; }
int av1pf_serve_submit(av1pf_server*, int32_t, const av1pf_request*, uint64_t*) { return AV1PF_ERR_UNSUPPORTED; }
int av1pf_serve_poll(av1pf_server*, uint64_t, int32_t, uint8_t*, double*) { return AV1PF_ERR_UNSUPPORTED; }
int av1pf_serve_stats_get(av1pf_server*, av1pf_serve_stats*) { return AV1PF_ERR_UNSUPPORTED; }
int av1pf_serve_close(av1pf_server*) { return AV1PF_OK; }
}
