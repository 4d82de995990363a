// msg_learned.cu -- learned Newton initial guess (placeholder until the CNN lands).
#include "msg_ctx.cuh"
namespace msg {
bool learned_ready(msg_ctx *c) { return false; }
int learned_guess(msg_ctx *c) { return MSG_ERR_STATE; }
void learned_free(msg_ctx *c) {}
}
