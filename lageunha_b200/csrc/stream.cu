// Streamed force evaluations: host copies overlapped with the evaluations.
//
// A caller that evaluates a sequence of particle sets from host memory (a
// stream of boxes, or the steps of a code that keeps its particles on the
// host, as the reference's pmmain/treecorrection callers do) pays two host
// copies per evaluation. Here each submission queues the copy of its
// positions on a copy-in stream, the evaluation on the context's stream and
// the copy of its forces on a copy-out stream, in one of two slots of
// device buffers, and returns: the copy-in of submission k+1 and the
// copy-out of submission k-1 run during the evaluation of submission k.
// Events order the slots: a slot's positions are overwritten only after the
// evaluation that read them, its forces only after their copy-out.
#include <string.h>

#include "ctx.cuh"

using namespace tpm;

namespace {

int ensure_slots(tpm_ctx *c, int64_t np) {
  auto &sp = c->sp;
  if (!sp.in) {
    CK(cudaStreamCreateWithFlags(&sp.in, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&sp.out, cudaStreamNonBlocking));
    for (int s = 0; s < 2; s++) {
      CK(cudaEventCreateWithFlags(&sp.ev_in[s], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&sp.ev_comp[s], cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&sp.ev_out[s], cudaEventDisableTiming));
    }
    CK(cudaMallocHost(&sp.herr, sizeof(uint32_t) * 16));
    memset(sp.herr, 0, sizeof(uint32_t) * 16);
  }
  if (np <= sp.cap) return 0;
  // nothing may be in flight while the slots are replaced
  CK(cudaStreamSynchronize(sp.in));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaStreamSynchronize(sp.out));
  for (int s = 0; s < 2; s++) {
    dfree(c->arena, sp.pos[s]);
    dfree(c->arena, sp.force[s]);
    sp.pos[s] = nullptr;
    sp.force[s] = nullptr;
  }
  sp.cap = 0;
  for (int s = 0; s < 2; s++) {
    CK(dmalloc(c->arena, &sp.pos[s], sizeof(uint32_t) * 3 * np));
    CK(dmalloc(c->arena, &sp.force[s], sizeof(float) * 3 * np));
  }
  sp.cap = np;
  return 0;
}

}  // namespace

void tpm::free_stream_state(tpm_ctx *c) {
  auto &sp = c->sp;
  if (sp.in) cudaStreamSynchronize(sp.in);
  if (sp.out) cudaStreamSynchronize(sp.out);
  for (int s = 0; s < 2; s++) {
    dfree(c->arena, sp.pos[s]);
    dfree(c->arena, sp.force[s]);
    if (sp.ev_in[s]) cudaEventDestroy(sp.ev_in[s]);
    if (sp.ev_comp[s]) cudaEventDestroy(sp.ev_comp[s]);
    if (sp.ev_out[s]) cudaEventDestroy(sp.ev_out[s]);
    sp.pos[s] = nullptr;
    sp.force[s] = nullptr;
    sp.ev_in[s] = sp.ev_comp[s] = sp.ev_out[s] = nullptr;
  }
  if (sp.herr) cudaFreeHost(sp.herr);
  if (sp.in) cudaStreamDestroy(sp.in);
  if (sp.out) cudaStreamDestroy(sp.out);
  sp.herr = nullptr;
  sp.in = sp.out = nullptr;
  sp.cap = 0;
}

extern "C" {

int tpm_stream_submit(tpm_ctx *c, int64_t np, const uint32_t *pos, float *forces, unsigned parts,
                      int64_t *ticket) {
  if (!c || !pos || !forces || np <= 0) return fail(TPM_E_ARG, "bad arguments to tpm_stream_submit");
  if ((parts & TPM_PART_ALL) == 0) return fail(TPM_E_ARG, "no force part requested");
  if (np > 0xffffffffll - 64) return fail(TPM_E_ARG, "np %lld too large", (long long)np);
  CK(cudaSetDevice(c->device));
  auto &sp = c->sp;
  int s = (int)(sp.next & 1);
  if (sp.pending[s])
    return fail(TPM_E_STATE, "two submissions are in flight: wait for ticket %lld first", (long long)sp.ticket[s]);
  int64_t cap0 = c->cap;
  int rc = ensure_slots(c, np);
  if (!rc) rc = ensure_particles_for(c, np);
  if (rc) return rc;
  // the particles loaded in the context stay loaded unless the buffers grew
  int64_t loaded_np = c->cap == cap0 ? c->np : 0;
  // copy-in, after the evaluation that last read this slot's positions
  CK(cudaStreamWaitEvent(sp.in, sp.ev_comp[s], 0));
  CK(cudaMemcpyAsync(sp.pos[s], pos, sizeof(uint32_t) * 3 * np, cudaMemcpyHostToDevice, sp.in));
  CK(cudaEventRecord(sp.ev_in[s], sp.in));
  // the evaluation, after its copy-in and after the copy-out of this slot's
  // previous forces
  CK(cudaStreamWaitEvent(c->st, sp.ev_in[s], 0));
  CK(cudaStreamWaitEvent(c->st, sp.ev_out[s], 0));
  uint32_t *loaded = c->pos;
  c->pos = sp.pos[s];
  c->np = np;
  rc = enqueue_forces(c, parts, c->st, false);
  if (!rc) rc = launch_finish_to(c, c->st, parts, sp.force[s]);
  c->pos = loaded;
  c->np = loaded_np;
  if (rc) return rc;
  CK(cudaMemcpyAsync(sp.herr + 8 * s, c->err, sizeof(uint32_t) * 8, cudaMemcpyDeviceToHost, c->st));
  CK(cudaEventRecord(sp.ev_comp[s], c->st));
  // copy-out
  CK(cudaStreamWaitEvent(sp.out, sp.ev_comp[s], 0));
  CK(cudaMemcpyAsync(forces, sp.force[s], sizeof(float) * 3 * np, cudaMemcpyDeviceToHost, sp.out));
  CK(cudaEventRecord(sp.ev_out[s], sp.out));
  // the context's own particles are not the streamed ones
  c->parts_valid = 0;
  sp.ticket[s] = sp.next;
  sp.pending[s] = true;
  if (ticket) *ticket = sp.next;
  sp.next++;
  return 0;
}

int tpm_stream_wait(tpm_ctx *c, int64_t ticket) {
  if (!c || ticket < 0) return fail(TPM_E_ARG, "bad arguments to tpm_stream_wait");
  auto &sp = c->sp;
  int s = (int)(ticket & 1);
  if (!sp.pending[s] || sp.ticket[s] != ticket) return fail(TPM_E_STATE, "ticket %lld is not in flight", (long long)ticket);
  CK(cudaSetDevice(c->device));
  CK(cudaEventSynchronize(sp.ev_out[s]));
  sp.pending[s] = false;
  uint32_t e = sp.herr[8 * s];
  if (e) {
    if (e & kErrNodeOverflow) return fail(TPM_E_OVERFLOW, "tree node capacity exceeded");
    if (e & kErrStackOverflow) return fail(TPM_E_OVERFLOW, "tree-walk stack overflow");
    if (e & kErrTmaTimeout) return fail(TPM_E_CUDA, "TMA load timed out in fda4");
    return fail(TPM_E_CUDA, "device error flags 0x%x", e);
  }
  return 0;
}

}  // extern "C"
