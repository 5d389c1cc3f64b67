// Entry points whose implementation lands in a later step.
#include "common.hpp"

using namespace gpuga;

extern "C" {
#define PENDING(name, ...)                         \
  int name(__VA_ARGS__) {                          \
    set_error(#name " is not implemented yet.");   \
    return GPUGA_ERR_UNSUPPORTED;                  \
  }
PENDING(gpuga_server_create, int, double, int, gpuga_server**)
PENDING(gpuga_server_submit, gpuga_server*, const char*, unsigned, int, int*)
PENDING(gpuga_server_submit_engine, gpuga_server*, gpuga_engine*, int, int, float, int, unsigned, int*)
PENDING(gpuga_server_poll, gpuga_server*, int, int*)
PENDING(gpuga_server_result, gpuga_server*, int, float*, float*)
PENDING(gpuga_server_cancel, gpuga_server*, int)
PENDING(gpuga_server_drain, gpuga_server*, double)
PENDING(gpuga_server_stats, gpuga_server*, double*)
PENDING(gpuga_server_destroy, gpuga_server*)
}
