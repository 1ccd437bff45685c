// engine_methods_f32.cu -- the IBM method-kernel launches for StoreF32S
// storage (see engine_methods.cuh).
#define COUPLB_METHODS_IMPL
#include "engine_methods.cuh"

namespace couplb {
template int launch_method<D2Q9, StoreF32S>(couplb_handle*, PassArgs<StoreF32S>&, int, bool, int);
template int launch_method<D3Q19, StoreF32S>(couplb_handle*, PassArgs<StoreF32S>&, int, bool, int);
}  // namespace couplb
