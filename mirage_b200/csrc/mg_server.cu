// Served form (continuous batching). Placeholder entry points until the server loop lands.
#include "../../include/mirage_b200.h"

extern "C" {
int mg_server_create(mg_index*, const mg_server_config*, mg_server** out) {
  if (out) *out = nullptr;
  return MG_ERR_LIMIT;
}
int mg_server_submit(mg_server*, const mg_batch*, uint64_t*) { return MG_ERR_INVAL; }
int mg_server_poll(mg_server*, uint64_t, mg_result*) { return MG_ERR_INVAL; }
int mg_server_wait(mg_server*, uint64_t, mg_result*, uint32_t) { return MG_ERR_INVAL; }
void mg_server_destroy(mg_server*) {}
}
