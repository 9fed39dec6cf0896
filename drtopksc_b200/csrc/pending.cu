// pending.cu -- entry points whose implementation lands in later files.
#include "../../include/drtopk.h"

extern "C" {
drtopk_status_t drtopk_server_create(drtopk_server_t* s, int, size_t, int) { if (s) *s = nullptr; return DRTOPK_EUNSUPPORTED; }
drtopk_status_t drtopk_server_destroy(drtopk_server_t) { return DRTOPK_OK; }
drtopk_status_t drtopk_server_submit(drtopk_server_t, const void*, drtopk_dtype_t, uint64_t, uint64_t, int, void*, int64_t*, uint64_t*) { return DRTOPK_EUNSUPPORTED; }
drtopk_status_t drtopk_server_poll(drtopk_server_t, drtopk_result_t*, int, int* c) { if (c) *c = 0; return DRTOPK_EUNSUPPORTED; }
drtopk_status_t drtopk_server_cancel(drtopk_server_t, uint64_t) { return DRTOPK_EUNSUPPORTED; }
drtopk_status_t drtopk_server_drain(drtopk_server_t, int) { return DRTOPK_EUNSUPPORTED; }
drtopk_status_t drtopk_server_usage(drtopk_server_t, size_t*, int*, int*) { return DRTOPK_EUNSUPPORTED; }
}
