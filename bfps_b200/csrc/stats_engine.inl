// Engine<T, N>::stats — field::compute_stats (bfps/cpp/field.cpp:984-1040)
// for one complex 3-vector field in the state layout: co-spectrum, then the
// unnormalised C2R into scratch (v2 is free between steps: every step
// rewrites it completely) and the real-space moments and histograms.
// Included by bfps_b200.cu after the Engine definition.

template <typename T, int N>
int Engine<T, N>::stats(bfg_ctx* c, int cfield, double max_est, int nbins, double* spec,
                        double* mom, int64_t* hist) {
    const size_t spec_n = (size_t)c->nshells * 9;
    // spectrum: SPEC_BLOCKS partials of spec_n doubles, then the result
    int spec_warps = SPEC_WARPS_MAX;
    while (spec_warps > 1 && (size_t)spec_warps * spec_n * 8 > (size_t)c->smem_optin) --spec_warps;
    if (spec_n * 8 > (size_t)c->smem_optin)
        return fail(c, BFG_EUNSUP, "%d shells do not fit the spectrum kernel's shared memory",
                    c->nshells);
    const size_t need = spec_n * 8 + (size_t)SPEC_BLOCKS * spec_n * 8 +
                        (size_t)STATS_BLOCKS * NQ * 8 + NQ * 8 + (size_t)nbins * 4 * 8;
    if (c->stats_ws_bytes < need) {
        if (c->stats_ws) cudaFree(c->stats_ws);
        c->stats_ws = nullptr;
        c->stats_ws_bytes = 0;
        CU(cudaMalloc(&c->stats_ws, need));
        c->stats_ws_bytes = need;
    }
    double* d_spec = (double*)c->stats_ws;
    double* d_spart = d_spec + spec_n;
    double* d_part = d_spart + (size_t)SPEC_BLOCKS * spec_n;
    double* d_mom = d_part + (size_t)STATS_BLOCKS * NQ;
    unsigned long long* d_hist = (unsigned long long*)(d_mom + NQ);
    CU(cudaMemsetAsync(d_hist, 0, (size_t)nbins * 4 * 8, c->stream));
    const KParams kp = kparams(c, 0.0);
    Prof pr0(c, K_STATS);
    const void* cptr = cfield == B_W0 ? c->w0 : (cfield == B_V1 ? c->v1 : c->wa);
    const size_t spec_smem = (size_t)spec_warps * spec_n * 8;
    CU(ensure_smem(spectrum_kernel<T, N>, spec_smem, c->device));
    spectrum_kernel<T, N><<<SPEC_BLOCKS, spec_warps * 32, spec_smem, c->stream>>>(
        kp, (const C*)cptr, c->nshells, c->dk, d_spart);
    int rc = after_launch(c, "spectrum");
    if (rc) return rc;
    spectrum_final<<<(unsigned)((spec_n + 255) / 256), 256, 0, c->stream>>>(d_spart, SPEC_BLOCKS,
                                                                          (int)spec_n, d_spec);
    if ((rc = after_launch(c, "spectrum_final"))) return rc;
    // real-space field into v2 (as [z][y][x][3] reals)
    if ((rc = col<CM_IZ_PLAIN>(c, self(c), 1, roles(cfield, B_NONE, B_WB, B_NONE)))) return rc;
    if ((rc = col<CM_Y_INV1>(c, self(c), 1, roles(B_WB, B_NONE, B_WB, B_NONE)))) return rc;
    if ((rc = row<RM_C2R, false>(c, self(c), 1, roles(B_WB, B_NONE, B_NONE, B_NONE, B_NONE,
                                                     B_NONE, B_NONE, B_V2))))
        return rc;
    const double me3 = max_est * std::sqrt(3.0);
    const size_t npts = (size_t)N * N * N;
    CU(ensure_smem(moments_kernel<T>, (size_t)nbins * 4 * 4, c->device));
    Prof pr1(c, K_STATS);
    moments_kernel<T><<<STATS_BLOCKS, STATS_THREADS, (size_t)nbins * 4 * 4, c->stream>>>(
        (const T*)c->v2, npts, max_est, max_est, max_est, me3, nbins, d_part, d_hist);
    if ((rc = after_launch(c, "moments"))) return rc;
    moments_final<<<1, 64, 0, c->stream>>>(d_part, STATS_BLOCKS, 1.0 / (double)npts, d_mom);
    if ((rc = after_launch(c, "moments_final"))) return rc;
    if (spec) CU(cudaMemcpyAsync(spec, d_spec, spec_n * 8, cudaMemcpyDeviceToHost, c->stream));
    if (mom) CU(cudaMemcpyAsync(mom, d_mom, NQ * 8, cudaMemcpyDeviceToHost, c->stream));
    if (hist) CU(cudaMemcpyAsync(hist, d_hist, (size_t)nbins * 4 * 8, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return 0;
}
