// serve.cu -- the serving loop (pcc_submit / pcc_poll).
#include "pcc_objects.h"

namespace pcc {

void server_shutdown(pcc_ctx* ctx) { (void)ctx; }

}  // namespace pcc
