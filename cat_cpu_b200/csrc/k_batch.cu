// k_batch.cu -- placeholder for the batched persistent path.
#include "../../include/ltl.h"
#include "ltl_kernels.h"
struct ltl_batch { int dummy; };
extern "C" int ltl_batch_create(ltl_batch** out, int, const ltl_grid_desc*, int, int) {
    if (out) *out = nullptr; ltl_set_error("batched path not built yet"); return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_destroy(ltl_batch*) { return LTL_OK; }
extern "C" int ltl_batch_set_stream(ltl_batch*, void*) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_upload(ltl_batch*, int, const uint8_t*, size_t) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_download(ltl_batch*, int, uint8_t*, size_t) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_upload_all(ltl_batch*, const uint8_t*) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_download_all(ltl_batch*, uint8_t*) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_step(ltl_batch*, int) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_synchronize(ltl_batch*) { return LTL_EUNSUPPORTED; }
extern "C" int ltl_batch_info(const ltl_batch*, long long*, long long*, int*) { return LTL_EUNSUPPORTED; }
