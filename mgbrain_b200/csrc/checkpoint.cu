// Checkpoints: the state a simulation continues from, to and from host memory.
#include "sim.h"

using namespace mgc;

extern "C" {

// ---- checkpoints -------------------------------------------------------------

namespace {

constexpr uint64_t kCheckpointMagic = 0x3230545043474d4dull;  // "MMGCPT02"

struct CheckpointHeader {
    uint64_t magic;
    int64_t n, ns, S;
    int32_t mode, M, H, D, stdp, ahead, fx, fx_shift;
    int32_t acc_mask, reserved;  // the accumulator cycle the buffers are laid out in
    int64_t bytes;               // whole checkpoint
};

struct Segment {
    void* dev;
    size_t bytes;
};

// The device state a step depends on, in a fixed order.
std::vector<Segment> state_segments(mgc_sim* s)
{
    StepArgs& a = s->a;
    const size_t ns = (size_t)a.ns, n = (size_t)s->n;
    const size_t acc = a.fx ? 8 : 4;  // accumulator entry: fp32 or 64-bit fixed point
    std::vector<Segment> v = {
        {a.V, 4 * ns}, {a.Iexc, 4 * ns}, {a.Iinh, 4 * ns}, {a.refrac, 4 * ns}, {a.last_fired, 4 * ns},
        {a.fire_cnt, 4 * ns}, {const_cast<float*>(a.rate), 4 * ns}, {a.step, 16}, {a.events, 8},
        {a.spk_count, 4}};
    if (a.deferred) {
        v.push_back({a.acc_e, acc * (size_t)s->acc_buffers * ns});
        v.push_back({a.acc_i, acc * (size_t)s->acc_buffers * ns});
        v.push_back({a.hist_ids, 4 * (size_t)a.H * (size_t)s->n_src});
        v.push_back({a.hist_cnt, 4 * (size_t)a.H});
    } else {
        v.push_back({a.ring_e, acc * (size_t)s->M * ns});
        v.push_back({a.ring_i, acc * (size_t)s->M * ns});
        v.push_back({a.spk, 4 * n});
    }
    if (s->stdp) v.push_back({a.pull ? (void*)a.in_ent : (void*)a.syn, 8 * (size_t)s->S});  // plastic weights
    return v;
}

CheckpointHeader checkpoint_header(mgc_sim* s)
{
    CheckpointHeader h{};
    h.magic = kCheckpointMagic;
    h.n = s->n;
    h.ns = s->a.ns;
    h.S = s->S;
    h.mode = s->mode;
    h.M = s->M;
    h.H = s->a.H;
    h.D = s->a.D;
    h.stdp = s->stdp;
    h.ahead = s->ahead;
    h.fx = s->a.fx;
    h.fx_shift = s->fx_shift;
    h.acc_mask = s->a.acc_mask;
    h.bytes = sizeof(CheckpointHeader);
    for (const Segment& g : state_segments(s)) h.bytes += (int64_t)g.bytes;
    return h;
}

}  // namespace

mgc_status mgc_checkpoint_size(mgc_sim* s, int64_t* bytes)
{
    if (!s || !bytes) return fail(MGC_ERR_INVALID, "null argument");
    *bytes = checkpoint_header(s).bytes;
    return MGC_OK;
}

mgc_status mgc_checkpoint_save(mgc_sim* s, void* buf, int64_t bytes)
{
    if (!s || !buf) return fail(MGC_ERR_INVALID, "null argument");
    if (s->partition && s->pending)
        return fail(MGC_ERR_INVALID, "partition: save a checkpoint right after an exchange");
    CK(cudaSetDevice(s->device));
    const CheckpointHeader h = checkpoint_header(s);
    if (bytes < h.bytes) return fail(MGC_ERR_INVALID, "checkpoint buffer of %lld bytes, need %lld", (long long)bytes,
                                     (long long)h.bytes);
    CK(cudaStreamSynchronize(s->stream));
    char* p = static_cast<char*>(buf);
    memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    for (const Segment& g : state_segments(s)) {
        CK(cudaMemcpy(p, g.dev, g.bytes, cudaMemcpyDeviceToHost));
        p += g.bytes;
    }
    return MGC_OK;
}

mgc_status mgc_checkpoint_load(mgc_sim* s, const void* buf, int64_t bytes)
{
    if (!s || !buf) return fail(MGC_ERR_INVALID, "null argument");
    CK(cudaSetDevice(s->device));
    CheckpointHeader h;
    if (bytes < (int64_t)sizeof(h)) return fail(MGC_ERR_INVALID, "not a checkpoint");
    memcpy(&h, buf, sizeof(h));
    const CheckpointHeader mine = checkpoint_header(s);
    if (h.magic != kCheckpointMagic) return fail(MGC_ERR_INVALID, "not a checkpoint");
    if (h.n != mine.n || h.S != mine.S || h.mode != mine.mode || h.M != mine.M || h.H != mine.H || h.D != mine.D ||
        h.stdp != mine.stdp || h.fx != mine.fx || h.fx_shift != mine.fx_shift || h.bytes != mine.bytes ||
        bytes < h.bytes || (s->a.deferred && h.acc_mask != kAccBuffers - 1 && h.acc_mask + 1 != s->acc_buffers))
        return fail(MGC_ERR_INVALID, "the checkpoint is of another network or method");
    CK(cudaStreamSynchronize(s->stream));
    const char* p = static_cast<const char*>(buf) + sizeof(h);
    for (const Segment& g : state_segments(s)) {
        CK(cudaMemcpy(g.dev, p, g.bytes, cudaMemcpyHostToDevice));
        p += g.bytes;
    }
    // the raster starts empty at the restored step; nothing is pending
    int64_t step = 0;
    const int64_t zero = 0;
    const int32_t zero32 = 0;
    CK(cudaMemcpy(&step, s->a.step, 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(s->a.raster_step0, &step, 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->a.raster_pos, &zero, 8, cudaMemcpyHostToDevice));
    if (s->a.bits_span) {  // the spike bitmaps of pull steps are not part of it
        const int64_t none[2] = {0, -1};
        CK(cudaMemcpy(s->a.bits_span, none, sizeof(none), cudaMemcpyHostToDevice));
    }
    CK(cudaMemcpy(s->a.status, &zero32, 4, cudaMemcpyHostToDevice));
    if (s->a.ev_mark) {
        unsigned long long ev = 0;
        CK(cudaMemcpy(&ev, s->a.events, 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(s->a.ev_mark, &ev, 8, cudaMemcpyHostToDevice));
    }
    s->ahead = h.ahead != 0;
    s->pending = 0;  // a partition's checkpoint is taken between exchanges
    CKS(set_acc_mask(s, h.acc_mask, false));  // the restored buffers' cycle
    return MGC_OK;
}

}  // extern "C"
