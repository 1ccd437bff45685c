// engine_methods_f64.cu -- the IBM method-kernel launches for StoreF64
// storage (see engine_methods.cuh).
#define COUPLB_METHODS_IMPL
#include "engine_methods.cuh"

namespace couplb {
template int launch_method<D2Q9, StoreF64>(couplb_handle*, PassArgs<StoreF64>&, int, bool, int);
template int launch_method<D3Q19, StoreF64>(couplb_handle*, PassArgs<StoreF64>&, int, bool, int);
}  // namespace couplb
