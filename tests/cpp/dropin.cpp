// C++17 drop-in check: code written against the reference's limbforge headers (Engine, Buffer,
// CommandBatch, Linalg, BatchedLinalg) compiles unchanged against include/limbforge/*.hpp and runs on
// the GPU through liblimbforge_b200.so.  Prints one line per check; exit status 0 when all pass.
#include "limbforge/batched_linalg.hpp"
#include "limbforge/exact_gemm4.hpp"
#include "limbforge/linalg.hpp"
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace limbforge;
template <int Bits> Float<Bits> power(int e, int sign = 1) { auto x = zero<Bits / 32>(); x.limb[Bits / 32 - 1] = 0x80000000u; x.sign = sign; x.exponent = e; return x; }

int main() {
    try {
        Engine e;
        std::printf("device %s\n", e.device_name().c_str());
        // 2^i * 2^1 = 2^(i+1), exactly, through a host-array call and a resident fused chain
        constexpr int B = 256;
        std::vector<Float<B>> a(64), b(64), out(64);
        for (int i = 0; i < 64; ++i) { a[i] = power<B>(i); b[i] = power<B>(1); }
        e.run(B, Operation::mul, a.data(), b.data(), out.data(), 64);
        for (int i = 0; i < 64; ++i) if (out[i].exponent != i + 1 || out[i].sign != 1) { std::printf("mul FAILED at %d\n", i); return 1; }
        auto x = e.make_buffer<Float<B>>(64), f = e.make_buffer<Float<B>>(64);
        x.upload(a.data(), 64); f.upload(b.data(), 64);
        auto batch = e.batch();
        for (int s = 0; s < 8; ++s) batch.run(Operation::mul, x, f, x);
        batch.submit().wait();
        x.download(out.data(), 64);
        for (int i = 0; i < 64; ++i) if (out[i].exponent != i + 8) { std::printf("chain FAILED at %d\n", i); return 1; }
        std::printf("engine ok\n");
        // cast 256 -> 1024 bits (exact) and the tree sum of 2^1..2^64: sum of powers, exactly representable
        auto wide = e.make_buffer<Float<1024>>(64), total = e.make_buffer<Float<1024>>(1);
        auto rb = e.batch();
        rb.cast(x, wide);
        rb.tree_sum(wide, total);
        rb.submit().wait();
        Float<1024> t{};
        total.download(&t, 1);
        // sum_{i=8}^{71} 2^i = 2^72 - 2^8: top bit 2^71, exponent 71, and the 1024-bit mantissa holds it exactly
        if (t.exponent != 71 || t.sign != 1 || t.limb[31] != 0xffffffffu || t.limb[30] != 0xffffffffu) { std::printf("cast/tree_sum FAILED\n"); return 1; }
        std::vector<Float<128>> narrow(64);
        e.cast(B, 128, false, a.data(), narrow.data(), 64);
        for (int i = 0; i < 64; ++i) if (narrow[i].exponent != i || narrow[i].limb[3] != 0x80000000u) { std::printf("host cast FAILED at %d\n", i); return 1; }
        std::printf("cast and tree_sum ok\n");
        // exact products: (A^T A) with A = identity-like powers
        Linalg la(e);
        std::vector<Float<B>> A(9, zero<B / 32>()), C(9);
        for (int i = 0; i < 3; ++i) A[i * 3 + i] = power<B>(i);
        la.syrk(B, A.data(), 3, 3, C.data(), false);
        for (int i = 0; i < 3; ++i) if (C[i * 3 + i].exponent != 2 * i) { std::printf("syrk FAILED\n"); return 1; }
        {   // the same SYRK resident in a batch: planned on the GPU, identical bits after wait
            auto bA = e.make_buffer<Float<B>>(9), bC = e.make_buffer<Float<B>>(9);
            bA.upload(A.data(), 9);
            auto rb = e.batch();
            LinalgTicket t = la.syrk(rb, bA, 3, 3, bC, false);
            rb.submit().wait();
            std::vector<Float<B>> C2(9);
            bC.download(C2.data(), 9);
            if (std::memcmp(C2.data(), C.data(), sizeof(Float<B>) * 9) || !t.resolved() || t.report().m != 3) {
                std::printf("resident syrk FAILED\n"); return 1;
            }
            std::printf("resident syrk ok\n");
        }
        std::vector<Float<B>> L(9);
        CholeskyInfo info = la.cholesky(B, C.data(), 3, L.data());
        if (info.pivot != 3 || L[4].exponent != 1) { std::printf("cholesky FAILED\n"); return 1; }
        {   // retained memory: the calls above left scratch; release frees it and later calls allocate afresh
            const LinalgWorkspaces w = la.workspaces();
            const LinalgWorkspaces r = la.release_workspaces();
            if (!w.scratch_bytes || r.scratch_bytes != w.scratch_bytes || la.workspaces().scratch_bytes) { std::printf("workspaces FAILED\n"); return 1; }
            std::vector<Float<B>> C3(9);
            la.syrk(B, A.data(), 3, 3, C3.data(), false);
            if (std::memcmp(C3.data(), C.data(), sizeof(Float<B>) * 9)) { std::printf("syrk after release FAILED\n"); return 1; }
        }
        std::printf("linalg ok\n");
        {   // the rest of the reference's public surface: prewarm, pipeline info, segmented dots, recurrences,
            // Buffer-form factorization and solves, the full report, host scalar arithmetic, version checks
            Prewarm pw; pw.bits = {64, 256}; pw.operations = {Operation::mul, Operation::complex_fma};
            e.prewarm(pw);
            e.prewarm_async(pw).get();
            const PipelineInfo pi = e.pipeline_info(256, Operation::mul);
            if (pi.simd_width != 32 || !pi.max_threads || !pi.threads_per_threadgroup) { std::printf("pipeline_info FAILED\n"); return 1; }
            LinalgPrewarm lp; lp.bits = {256}; lp.inner_sizes = {32};
            la.prewarm(lp);
            la.prewarm_async(lp).get();
            if (la.device_name().empty()) { std::printf("linalg device_name FAILED\n"); return 1; }
            SegmentedDot sd; sd.segments = 2; sd.length = 3;
            std::vector<Float<B>> da(6, power<B>(1)), db(6, power<B>(2)), dout(2);
            e.segmented_dot(B, false, sd, da.data(), db.data(), dout.data());       // 3 * 2^3 = 2^4 + 2^3
            if (dout[0].exponent != 4 || dout[1].limb[B / 32 - 1] != 0xC0000000u) { std::printf("segmented_dot FAILED\n"); return 1; }
            auto ba = e.make_buffer<Float<B>>(6), bb = e.make_buffer<Float<B>>(6), bo = e.make_buffer<Float<B>>(2);
            ba.upload(da.data(), 6); bb.upload(db.data(), 6);
            auto sb = e.batch();
            sb.segmented_dot(sd, ba, bb, bo);
            sb.submit().wait();
            std::vector<Float<B>> dout2(2);
            bo.download(dout2.data(), 2);
            if (std::memcmp(dout2.data(), dout.data(), sizeof(Float<B>) * 2)) { std::printf("batch segmented_dot FAILED\n"); return 1; }
            // ring (1, 1, 1, 1) with weights (1, 0, 0, 0): each step moves q0 to the end, so the result is 1
            std::vector<Complex<B / 32>> seeds(4, {power<B>(0), zero<B / 32>()}), w(4, {zero<B / 32>(), zero<B / 32>()}), q(1);
            w[0] = {power<B>(0), zero<B / 32>()};
            e.recurrence(B, seeds.data(), w.data(), q.data(), 1, 1);
            if (q[0].re.exponent != 0 || q[0].re.sign != 1 || q[0].im.sign) { std::printf("recurrence FAILED\n"); return 1; }
            bool vr = false;
            try { e.vector_recurrence(B, VectorRecurrence{}, nullptr, nullptr, nullptr, nullptr, nullptr); } catch (const std::runtime_error&) { vr = true; }
            if (!vr) { std::printf("vector_recurrence FAILED\n"); return 1; }
            auto bA = e.make_buffer<Float<B>>(9), bL = e.make_buffer<Float<B>>(9), bR = e.make_buffer<Float<B>>(3), bX = e.make_buffer<Float<B>>(3);
            bA.upload(C.data(), 9);
            const CholeskyInfo bi = la.cholesky(bA, 3, bL);
            std::vector<Float<B>> L2(9);
            bL.download(L2.data(), 9);
            if (bi.pivot != 3 || std::memcmp(L2.data(), L.data(), sizeof(Float<B>) * 9)) { std::printf("buffer cholesky FAILED\n"); return 1; }
            std::vector<Float<B>> rhs = {power<B>(0), power<B>(2), power<B>(4)}, X1(3), X2(3);
            bR.upload(rhs.data(), 3);
            la.cholesky_solve(B, L.data(), 3, rhs.data(), 1, X1.data());
            la.cholesky_solve(bL, 3, bR, 1, bX);
            bX.download(X2.data(), 3);
            if (std::memcmp(X1.data(), X2.data(), sizeof(Float<B>) * 3)) { std::printf("buffer cholesky_solve FAILED\n"); return 1; }
            la.trsm(false, bL, 3, bR, 1, bX);
            la.cholesky_blocked(bA, 3, bL);
            la.cholesky_solve_blocked(bL, 3, bR, 1, bX);
            std::vector<Float<B>> G(4 * 3, power<B>(0)), P(9);
            la.syrk(B, G.data(), 4, 3, P.data(), false);
            const LinalgReport& rep = la.report();
            if (rep.left_bands.size() != 2 || rep.left_bands[1] != 3 || rep.left_fallback || rep.fallback_outputs) { std::printf("report FAILED\n"); return 1; }
            const Float<B> s = add(power<B>(3), power<B>(3)), p = mul(power<B>(3), power<B>(-5)), f = fma(power<B>(1), power<B>(1), power<B>(2));
            if (s.exponent != 4 || p.exponent != -2 || f.exponent != 3 || magnitude_compare(s, p) <= 0) { std::printf("host arithmetic FAILED\n"); return 1; }
            std::vector<Float<B>> xs(3, power<B>(1)), ys(3, power<B>(1));
            if (exact_dot(xs.data(), 1, ys.data(), 1, 3).limb[B / 32 - 1] != 0xC0000000u) { std::printf("exact_dot FAILED\n"); return 1; }
            {   // Householder QR of diag(2, 2) stacked on a zero row: R = diag(2, 2), Q = I; least squares of (2, 4, 0) is (1, 2)
                std::vector<Float<B>> qa = {power<B>(1), zero<B / 32>(), zero<B / 32>(), power<B>(1), zero<B / 32>(), zero<B / 32>()};
                QROptions qopt;
                qopt.block = 1;
                QRFactor qf = la.factor_qr(B, qa.data(), 3, 2, qopt);
                std::vector<Float<B>> qb = {power<B>(1), power<B>(2), zero<B / 32>()}, qx(2), qb0 = qb;
                qf.solve(qb.data(), 1, qx.data());
                if (!qf.full_rank() || qf.rows() != 3 || qf.cols() != 2 || qf.info().reason != QRInfo::full_rank || qx[0].exponent != 0 ||
                    qx[1].exponent != 1) { std::printf("qr solve FAILED\n"); return 1; }
                qf.apply_q(qb.data(), 1, true);
                if (qb[1].exponent != 2) { std::printf("qr apply_q FAILED\n"); return 1; }
                auto bq = e.make_buffer<Float<B>>(6);
                bq.upload(qa.data(), 6);
                QRFactor qg = la.factor_qr(bq, 3, 2, qopt);
                if (std::memcmp(qg.r(), qf.r(), sizeof(Float<B>) * 4)) { std::printf("buffer qr FAILED\n"); return 1; }
                QRFactor qm = std::move(qg);
                if (!qg.empty() || qm.empty() || qm.pivoted() || qm.permutation()[1] != 1) { std::printf("qr move FAILED\n"); return 1; }
                std::vector<Float<B>> dd(2, power<B>(0));
                if (la.factor_qr_augmented(B, qa.data(), 3, 2, dd.data(), qopt).rows() != 5) { std::printf("augmented qr FAILED\n"); return 1; }
                // complex: the same matrix with zero imaginary parts gives the real factor in the real parts
                std::vector<Complex<B / 32>> ca(6), cb(3), cx(2);
                for (int i = 0; i < 6; ++i) ca[i] = {qa[i], zero<B / 32>()};
                for (int i = 0; i < 3; ++i) cb[i] = {qb0[i], zero<B / 32>()};
                ComplexQRFactor cq = la.factor_qr_complex(B, ca.data(), 3, 2, qopt);
                cq.solve(cb.data(), 1, cx.data());
                if (!cq.full_rank() || cx[0].re.exponent != 0 || cx[1].re.exponent != 1 || cx[0].im.sign || cx[1].im.sign) {
                    std::printf("complex qr FAILED\n"); return 1;
                }
                cq.apply_q(cb.data(), 1, true);
            }
            check_library_version();
            if (!version_compatible(library_version(), header_version) || std::string(library_version_string()).empty()) { std::printf("version FAILED\n"); return 1; }
            std::printf("full surface ok\n");
        }
        BatchedLinalg bl(e);
        StridedGemm s; s.count = 1; s.m = s.n = s.k = 2; s.stride_a = s.stride_b = s.stride_c = 4;
        std::vector<Complex<B / 32>> ca(4), cb(4), cc(4);
        for (auto& z : ca) z = {power<B>(0), zero<B / 32>()};
        for (auto& z : cb) z = {power<B>(1), zero<B / 32>()};
        bl.gemm(B, true, s, ca.data(), cb.data(), cc.data());
        if (cc[0].re.exponent != 2) { std::printf("batched gemm FAILED\n"); return 1; }
        {   // (A B) D through product3's intermediate: ones x twos = 4 per entry, times ones = 8 = 2^3
            auto bA = e.make_buffer<Complex<B / 32>>(4), bB = e.make_buffer<Complex<B / 32>>(4);
            auto bD = e.make_buffer<Complex<B / 32>>(4), bC = e.make_buffer<Complex<B / 32>>(4);
            bA.upload(ca.data(), 4); bB.upload(cb.data(), 4); bD.upload(ca.data(), 4);
            auto pb = e.batch();
            bl.product3(pb, s, s, bA, bB, bD, bC);
            if (bl.workspaces().busy_workspaces != 1) { std::printf("product3 workspace FAILED\n"); return 1; }
            pb.submit().wait();
            std::vector<Complex<B / 32>> c3(4);
            bC.download(c3.data(), 4);
            for (auto& z : c3) if (z.re.exponent != 3 || z.im.sign != 0) { std::printf("product3 FAILED\n"); return 1; }
            const BatchedWorkspaces w = bl.workspaces();
            if (w.busy_workspaces || !w.idle_bytes || bl.release_workspaces().idle_bytes != w.idle_bytes || bl.workspaces().idle_bytes) {
                std::printf("batched workspaces FAILED\n"); return 1;
            }
        }
        std::printf("batched ok\n");
        {   // exact 4x4: I * 2 = 2 everywhere; accumulated onto itself and negated: -4; resident form with a ticket
            wolfnum::experimental::ExactGemm4 g(e);
            std::vector<Float<B>> I4(16, zero<B / 32>()), T4(16, power<B>(1)), C4(16);
            for (int i = 0; i < 4; ++i) I4[i * 5] = power<B>(0);
            wolfnum::experimental::ExactGemm4Shape gs;
            wolfnum::experimental::ExactGemm4Report gr;
            g.gemm(B, false, gs, I4.data(), T4.data(), C4.data(), &gr);
            gs.accumulate = gs.negative = true;
            g.gemm(B, false, gs, I4.data(), T4.data(), C4.data());
            for (auto& x : C4) if (x.exponent != 2 || x.sign != -1) { std::printf("exact gemm4 FAILED\n"); return 1; }
            if (gr.gpu_components != 16 || gr.host_components) { std::printf("exact gemm4 report FAILED\n"); return 1; }
            auto gA = e.make_buffer<Float<B>>(16), gB = e.make_buffer<Float<B>>(16), gC = e.make_buffer<Float<B>>(16);
            gA.upload(I4.data(), 16); gB.upload(T4.data(), 16); gC.upload(C4.data(), 16);
            auto gb = e.batch();
            auto ticket = g.gemm(gb, gs, gA, gB, gC);                 // -(-4 + 2) = 2
            if (ticket.resolved()) { std::printf("exact gemm4 ticket FAILED\n"); return 1; }
            gb.submit().wait();
            gC.download(C4.data(), 16);
            for (auto& x : C4) if (x.exponent != 1 || x.sign != 1) { std::printf("resident exact gemm4 FAILED\n"); return 1; }
            if (!ticket.resolved() || ticket.report().gpu_components != 16) { std::printf("exact gemm4 ticket FAILED\n"); return 1; }
        }
        std::printf("exact gemm4 ok\n");
        bool threw = false;
        try { e.run(100, Operation::add, a.data(), b.data(), out.data(), 1); } catch (const std::invalid_argument&) { threw = true; }
        if (!threw) { std::printf("error mapping FAILED\n"); return 1; }
        std::printf("all drop-in checks passed\n");
        return 0;
    } catch (const std::exception& ex) {
        std::printf("exception: %s\n", ex.what());
        return 1;
    }
}
