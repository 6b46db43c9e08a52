// Servo filter on the device (lib/servo.c servo_new / servo_filter /
// servo_reset): the DM-command integrator downstream of the reconstruction
// (maos/filter.c filter_dm), for n command values (e.g. nbatch instances x
// nact actuators) stepping together.  FP64 state, elementwise.
//
// One step, as servo_filter:
//   1. delay: with al > 0 the error used is the one given al steps earlier
//      (a FIFO of al+1 slots, servo_shift_al); before that, no update;
//   2. history: mint[0] <- sum_i ap[i] mint[i], older entries shift down one
//      (servo_shift_ap, ap padded to at least 2 terms);
//   3. pre-integrator: type I (ep 1 x 1 or 1 x n): ep .* merr;
//      PID (ep 2 x 1): (ep0+ep1) merr - ep1 merr_last;
//      type II (ep 3 x 1 or 3 x n; gain, a, T converted as servo_update to
//      gain, exp(-dt/(aT)), exp(-dt/T)): mlead = e1a mlead + g (1-e1a)/(1-e1)
//      (merr - e1 merr_last), and mpreint += mlead;
//   4. mint[0] += mpreint.
// The command is mint[0].  Products and sums are rounded separately
// (__dmul_rn/__dadd_rn) in the reference's order, so the device follows the
// reference's FP64 arithmetic.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"

namespace mb {

constexpr int kServoMaxAp = 8;

struct ServoParams {
    int nap, type, per_mode;  // type: 1 (type I), 2 (PID), 3 (type II)
    double ap[kServoMaxAp];
    int slot[kServoMaxAp];    // ring slot of mint[k] before this step
};

// grid: ceil(n/256).  hwrite / hread: the delay FIFO's slots for this step's
// error and for the one al steps old; update: that error exists; m0: the
// ring slot that takes the new mint[0] (the oldest entry's).
__global__ void k_servo_step(const double *__restrict__ merr, double *__restrict__ hist, double *__restrict__ mint,
                             double *__restrict__ pre, double *__restrict__ last, double *__restrict__ lead,
                             const double *__restrict__ ep, double *__restrict__ cmd, long n, ServoParams P, int al,
                             int hwrite, int hread, int update, int m0) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double e = merr[i];
    if (al > 0) {  // 1. delay FIFO
        hist[(size_t)hwrite * n + i] = e;
        e = hist[(size_t)hread * n + i];
    }
    if (!update) {  // no error al steps old yet: the command stays
        cmd[i] = mint[(size_t)P.slot[0] * n + i];
        return;
    }
    // 2. integrator history: the new mint[0] from the old entries, last term first
    double m[kServoMaxAp];
#pragma unroll
    for (int k = 0; k < kServoMaxAp; k++)
        if (k < P.nap) m[k] = mint[(size_t)P.slot[k] * n + i];
    double c = __dmul_rn(m[P.nap - 1], P.ap[P.nap - 1]);
#pragma unroll
    for (int k = kServoMaxAp - 2; k >= 0; k--)
        if (k < P.nap - 1) c = __dadd_rn(c, __dmul_rn(m[k], P.ap[k]));
    // 3. pre-integrator
    double pr;
    if (P.type == 1) {
        pr = __dmul_rn(e, ep[P.per_mode ? i % P.per_mode : 0]);
    } else if (P.type == 2) {
        const double g1 = __dadd_rn(ep[0], ep[1]), g2 = -ep[1];
        pr = __dadd_rn(__dmul_rn(e, g1), __dmul_rn(last[i], g2));
        last[i] = e;
    } else {
        const long im = P.per_mode ? i % P.per_mode : 0;
        const double gg = ep[3 * im], e1a = ep[3 * im + 1], e1 = ep[3 * im + 2];
        const double lv = __dadd_rn(__dmul_rn(e1a, lead[i]),
                                    __dmul_rn(__ddiv_rn(__dmul_rn(gg, __dadd_rn(1.0, -e1a)), __dadd_rn(1.0, -e1)),
                                              __dadd_rn(e, -__dmul_rn(e1, last[i]))));
        lead[i] = lv;
        last[i] = e;
        pr = __dadd_rn(pre[i], lv);
    }
    pre[i] = pr;
    // 4. the command
    const double v = __dadd_rn(c, pr);
    mint[(size_t)m0 * n + i] = v;
    cmd[i] = v;
}

struct Servo {
    long n = 0;
    int al = 0, nmode = 0;
    ServoParams P{};
    DevBuf<double> hist, mint, pre, last, lead, ep;
    long step = 0;  // errors received (the delay FIFO's clock)
};

}  // namespace mb

struct mb_servo {
    mb::Servo S;
};

extern "C" {

int mb_servo_create(long n, const double *ap, int nap, int al, const double *ep, int ep_nx, int ep_ny, double dt,
                    mb_servo **out) {
    if (!out || n <= 0 || al < 0 || !ep || ep_nx < 1 || ep_nx > 3 || ep_ny < 1 || nap < 0 || nap > mb::kServoMaxAp ||
        (nap > 0 && !ap) || (ep_nx == 2 && ep_ny != 1) || (ep_ny > 1 && n % ep_ny)) {
        mb::set_error("mb_servo_create: invalid arguments");
        return MB_EINVAL;
    }
    *out = nullptr;
    mb_servo *h = new (std::nothrow) mb_servo();
    if (!h) return MB_ENOMEM;
    try {
        mb::Servo &S = h->S;
        S.n = n;
        S.al = al;
        // servo_new: ap defaults to {1}; at least 2 entries keep the history
        std::vector<double> a = nap ? std::vector<double>(ap, ap + nap) : std::vector<double>{1.0};
        if (a.size() < 2) a.resize(2, 0.0);
        S.P.nap = (int)a.size();
        for (int k = 0; k < S.P.nap; k++) S.P.ap[k] = a[k];
        S.P.type = ep_nx;
        S.P.per_mode = ep_ny > 1 ? ep_ny : 0;
        std::vector<double> e(ep, ep + (size_t)ep_nx * ep_ny);
        if (ep_nx == 3)  // servo_update: (gain, a, T) -> (gain, exp(-dt/(aT)), exp(-dt/T))
            for (int i = 0; i < ep_ny; i++) {
                const double A = e[1 + 3 * i], T = e[2 + 3 * i];
                e[1 + 3 * i] = std::exp(-dt / (A * T));
                e[2 + 3 * i] = std::exp(-dt / T);
            }
        S.ep.upload(e);
        S.hist.alloc((size_t)(al + 1) * n);
        S.mint.alloc((size_t)S.P.nap * n);
        S.pre.alloc(n);
        S.last.alloc(n);
        S.lead.alloc(n);
        for (int k = 0; k < S.P.nap; k++) S.P.slot[k] = k;
        S.hist.zero_async(nullptr);
        S.mint.zero_async(nullptr);
        S.pre.zero_async(nullptr);
        S.last.zero_async(nullptr);
        S.lead.zero_async(nullptr);
        MB_CUDA_TRY(cudaDeviceSynchronize());
    } catch (const mb::CudaError &e) {
        delete h;
        return e.code;
    }
    *out = h;
    return MB_OK;
}

void mb_servo_free(mb_servo *h) { delete h; }

int mb_servo_reset(mb_servo *h) {
    if (!h) return MB_EINVAL;
    try {
        mb::Servo &S = h->S;
        S.step = 0;
        for (int k = 0; k < S.P.nap; k++) S.P.slot[k] = k;
        S.hist.zero_async(nullptr);
        S.mint.zero_async(nullptr);
        S.pre.zero_async(nullptr);
        S.last.zero_async(nullptr);
        S.lead.zero_async(nullptr);
        MB_CUDA_TRY(cudaDeviceSynchronize());
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

int mb_servo_filter(mb_servo *h, const double *d_merr, double *d_cmd, void *stream) {
    if (!h || !d_merr || !d_cmd) {
        mb::set_error("mb_servo_filter: invalid arguments");
        return MB_EINVAL;
    }
    try {
        mb::Servo &S = h->S;
        const int R = S.al + 1;
        // FIFO: this step's error into slot step % R; the one al steps old is
        // in slot (step + 1) % R once al errors came before it
        const int hw = (int)(S.step % R), hr = (int)((S.step + 1) % R);
        const bool update = S.step >= S.al;
        const int m0 = S.P.slot[S.P.nap - 1];  // the oldest history entry's slot takes the new mint[0]
        mb::k_servo_step<<<(unsigned)((S.n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
            d_merr, S.hist.p, S.mint.p, S.pre.p, S.last.p, S.lead.p, S.ep.p, d_cmd, S.n, S.P, S.al, hw, hr,
            update ? 1 : 0, m0);
        MB_CHECK_LAUNCH();
        if (update) {  // mint[k] <- mint[k-1]: rotate the slot table
            for (int k = S.P.nap - 1; k > 0; k--) S.P.slot[k] = S.P.slot[k - 1];
            S.P.slot[0] = m0;
        }
        S.step++;
    } catch (const mb::CudaError &e) {
        return e.code;
    }
    return MB_OK;
}

}  // extern "C"
