// Placement session (filled in by the pipeline engine).
#include "context.hpp"

namespace spk {
void session_destroy(spk_context* ctx) { ctx->session = nullptr; }
}  // namespace spk
