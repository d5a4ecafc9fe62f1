// shard.cpp -- one batch of profiles spread over several contexts (one per GPU).
//
// forward_model has no multi-device path in the reference (its profile loop is
// sequential, src/Sensor/sounder.jl:283-307); profiles are independent, so a batch is
// split into contiguous shards, one per context, each run by its own host thread on
// its own device, and the shards' channel spectra land in the caller's host buffers at
// their batch offsets (the gather needs no copy beyond each shard's own).  There is no
// collective on this path.
#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "irs_internal.h"

namespace {

// contiguous balanced shards: the first n % k shards take one profile more
void shard_of(int64_t n, int k, int i, int64_t& first, int64_t& count) {
    const int64_t q = n / k, r = n % k;
    first = i * q + std::min<int64_t>(i, r);
    count = q + (i < r ? 1 : 0);
}

}  // namespace

extern "C" int irs_shard_range(int64_t n, int n_shards, int shard, int64_t* first, int64_t* count) {
    if (n < 0 || n_shards < 1 || shard < 0 || shard >= n_shards || !first || !count) {
        irs::set_error("irs_shard_range: need n >= 0, n_shards >= 1, 0 <= shard < n_shards");
        return IRS_E_ARG;
    }
    shard_of(n, n_shards, shard, *first, *count);
    return IRS_OK;
}

extern "C" int irs_forward_model_batch_multi(irs_ctx* const* ctxs, int n_ctx, const irs_profile* profs, int n_prof,
                                             const irs_sounder* s, const irs_fm_options* o, double* R, double* BT) {
    if (!ctxs || n_ctx < 1 || !profs || n_prof < 1 || !s || !o || !R || !BT) {
        irs::set_error("irs_forward_model_batch_multi: invalid arguments");
        return IRS_E_ARG;
    }
    for (int k = 0; k < n_ctx; ++k) {
        if (!ctxs[k]) {
            irs::set_error("irs_forward_model_batch_multi: context " + std::to_string(k) + " is NULL");
            return IRS_E_ARG;
        }
        for (int j = 0; j < k; ++j)  // a context serves one host thread at a time
            if (ctxs[j] == ctxs[k]) {
                irs::set_error("irs_forward_model_batch_multi: context " + std::to_string(k) +
                               " repeats context " + std::to_string(j) + " (each context may appear once)");
                return IRS_E_ARG;
            }
    }
    const int64_t n_ch = irs::make_grid(s->nu_min, s->nu_max, s->dnu).n;  // as irs_forward_model_batch
    std::vector<int> rc(n_ctx, IRS_OK);
    std::vector<std::string> msg(n_ctx);
    auto run = [&](int k) {
        int64_t first = 0, count = 0;
        shard_of(n_prof, n_ctx, k, first, count);
        if (count == 0) return;
        rc[k] = irs_forward_model_batch(ctxs[k], profs + first, (int)count, s, o, R + first * n_ch,
                                        BT + first * n_ch);
        if (rc[k] != IRS_OK) msg[k] = irs_last_error();  // the message is per host thread
    };
    std::vector<std::thread> th;
    for (int k = 1; k < n_ctx; ++k) th.emplace_back(run, k);
    run(0);
    for (auto& t : th) t.join();
    for (int k = 0; k < n_ctx; ++k)
        if (rc[k] != IRS_OK) {
            irs::set_error("context " + std::to_string(k) + ": " + msg[k]);
            return rc[k];
        }
    return IRS_OK;
}
