// Problem setup on the device: TopologicalDOF::buildConstraints (topology/TopologicalDOF.tpp:34-111)
// and Assembler::createMatrix's pattern (fem/assembly/backend/cpu/Assembler.tpp:8-76), for meshes
// whose host build (one pass over the faces, a sort per row) would take seconds.
//
//   DOF map:  one thread per element face marks the nodes of faces on an essential tag with the
//             face's position e * faces + f + 1 by atomicMax, so a node keeps the last face in
//             element-then-face order that marked it, as the reference's loop does; free nodes are
//             numbered in node order by an exclusive scan (Interleaved ordering).
//   pattern:  a node -> element incidence by counting sort; then one warp per free row gathers the
//             free columns of every element touching the row's node into shared memory, keeps the
//             first occurrence of each column and places it by the number of smaller first
//             occurrences (sorted, unique, as the reference's per-row sort and unique), once to count
//             and once to fill after a scan of the counts.
// Rows with more candidate columns than a warp's buffer holds (kCand) are left to the host build.
#include <vector>

#include "rsd_kernels.cuh"

namespace rsd {
namespace {

constexpr int kScanItems = 4;                 // entries per thread of a scan block
constexpr int kScanThreads = 512;
constexpr int kScanBlock = kScanItems * kScanThreads;
constexpr int kRowWarpsSetup = 4;             // warps per block of the row kernels
constexpr int kCand = 512;                    // candidate columns a row may gather

// per block: exclusive scan of its kScanBlock counts (local offsets) and the block's total
__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(int64_t n, const int32_t* __restrict__ in, int32_t* __restrict__ out,
                                                              int64_t* __restrict__ sums) {
	__shared__ int32_t warpTot[kScanThreads / 32];
	const int64_t base = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanItems;
	int32_t v[kScanItems], t = 0;
#pragma unroll
	for (int k = 0; k < kScanItems; ++k) {
		v[k] = base + k < n ? in[base + k] : 0;
		t += v[k];
	}
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int32_t incl = t;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		const int32_t u = __shfl_up_sync(0xffffffffu, incl, o);
		if (lane >= o) incl += u;
	}
	if (lane == 31) warpTot[warp] = incl;
	__syncthreads();
	if (warp == 0) {
		int32_t w = lane < kScanThreads / 32 ? warpTot[lane] : 0;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const int32_t u = __shfl_up_sync(0xffffffffu, w, o);
			if (lane >= o) w += u;
		}
		if (lane < kScanThreads / 32) warpTot[lane] = w;   // inclusive over warps
	}
	__syncthreads();
	int32_t run = incl - t + (warp ? warpTot[warp - 1] : 0);
#pragma unroll
	for (int k = 0; k < kScanItems; ++k) {
		if (base + k < n) out[base + k] = run;
		run += v[k];
	}
	if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = (int64_t)run;
}

__global__ void k_scan_add(int64_t n, const int64_t* __restrict__ off, int32_t* __restrict__ out) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
		out[i] += (int32_t)off[i / kScanBlock];
}

// exclusive scan of n non-negative counts into out[0..n], out[n] = the total (< 2^31)
int exclusive_scan(rsd_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, int64_t* total) {
	const int64_t nb = std::max<int64_t>(1, (n + kScanBlock - 1) / kScanBlock);
	int64_t* sums = nullptr;
	RSD_CUDA(cudaMalloc(&sums, sizeof(int64_t) * nb));
	auto run = [&]() -> int {
		if (n) k_scan_blocks<<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(n, in, out, sums);
		RSD_CUDA(cudaGetLastError());
		std::vector<int64_t> h(nb, 0);
		if (n) RSD_CUDA(cudaMemcpyAsync(h.data(), sums, sizeof(int64_t) * nb, cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		int64_t acc = 0;
		for (int64_t b = 0; b < nb; ++b) { const int64_t s = h[b]; h[b] = acc; acc += s; }
		if (acc > INT32_MAX) return set_error(RSD_EINVAL, "a count exceeds 2^31 entries");
		*total = acc;
		RSD_CUDA(cudaMemcpyAsync(sums, h.data(), sizeof(int64_t) * nb, cudaMemcpyHostToDevice, ctx->stream));
		if (n) k_scan_add<<<vec_grid(ctx, n), 256, 0, ctx->stream>>>(n, sums, out);
		const int32_t t32 = (int32_t)acc;
		RSD_CUDA(cudaMemcpyAsync(out + n, &t32, sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
		RSD_CUDA(cudaGetLastError());
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		return RSD_OK;
	};
	const int rc = run();
	cudaFree(sums);
	return rc;
}

struct FaceTable {
	int32_t count;            // nodes per face
	int32_t node[6][16];      // element-local nodes of face f (LagrangeQuad/Hex::getFaceNodes order)
};

// win[node] = max over the faces on an essential tag that contain it of e * nf + f + 1
__global__ void k_mark_constrained(int64_t nelem, int nf, int npe, const int32_t* __restrict__ rng, const int32_t* __restrict__ ien,
                                   const int32_t* __restrict__ essTags, int nEss, FaceTable ft, uint32_t* __restrict__ win) {
	const int64_t total = nelem * nf;
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
		const int32_t tag = rng[i];
		if (tag < 0) continue;
		bool ess = false;
		for (int k = 0; k < nEss; ++k) ess |= essTags[k] == tag;
		if (!ess) continue;
		const int64_t e = i / nf;
		const int f = (int)(i - e * nf);
		for (int a = 0; a < ft.count; ++a) atomicMax(win + ien[e * npe + ft.node[f][a]], (uint32_t)(i + 1));
	}
}

// free[node] = 1 for unmarked nodes; ctag[node] = the expression index of the winning face's tag
__global__ void k_dof_flags(int64_t nn, const uint32_t* __restrict__ win, const int32_t* __restrict__ rng,
                            const int32_t* __restrict__ essTags, int nEss, int32_t* __restrict__ isFree, int32_t* __restrict__ ctag) {
	for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nn; v += (int64_t)gridDim.x * blockDim.x) {
		const uint32_t w = win[v];
		isFree[v] = w == 0;
		int32_t c = -1;
		if (w) {
			const int32_t tag = rng[w - 1];
			for (int k = 0; k < nEss; ++k)
				if (essTags[k] == tag) c = k;   // the last registration of a tag holds its expression
		}
		ctag[v] = c;
	}
}

// t2a[v] = scan[v] for free nodes, -1 otherwise; a2t[t2a[v]] = v
__global__ void k_dof_number(int64_t nn, const int32_t* __restrict__ isFree, const int32_t* __restrict__ scan,
                             int32_t* __restrict__ t2a, int32_t* __restrict__ a2t) {
	for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nn; v += (int64_t)gridDim.x * blockDim.x) {
		const int32_t r = isFree[v] ? scan[v] : -1;
		t2a[v] = r;
		if (r >= 0) a2t[r] = (int32_t)v;
	}
}

__global__ void k_incidence_count(int64_t total, const int32_t* __restrict__ ien, int32_t* __restrict__ cnt) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
		atomicAdd(cnt + ien[i], 1);
}
__global__ void k_incidence_fill(int64_t total, int npe, const int32_t* __restrict__ ien, int32_t* __restrict__ cur,
                                 int32_t* __restrict__ inc) {
	for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x)
		inc[atomicAdd(cur + ien[i], 1)] = (int32_t)(i / npe);
}

// One warp per free row: FILL = false writes the row's number of distinct free columns to cnt,
// FILL = true writes them sorted at col[rp[row]..].  err is raised when a row gathers more than kCand
// candidates.
template <bool FILL>
__global__ void __launch_bounds__(32 * kRowWarpsSetup) k_row_columns(int64_t n, int npe, const int32_t* __restrict__ a2t,
                                                                      const int32_t* __restrict__ ioff, const int32_t* __restrict__ inc,
                                                                      const int32_t* __restrict__ ien, const int32_t* __restrict__ t2a,
                                                                      int32_t* __restrict__ cnt, const int32_t* __restrict__ rp,
                                                                      int32_t* __restrict__ col, int32_t* __restrict__ err) {
	__shared__ int32_t cand[kRowWarpsSetup][kCand];
	__shared__ uint8_t first[kRowWarpsSetup][kCand];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	int32_t* c = cand[warp];
	uint8_t* fl = first[warp];
	for (int64_t row = (int64_t)blockIdx.x * kRowWarpsSetup + warp; row < n; row += (int64_t)gridDim.x * kRowWarpsSetup) {
		const int32_t node = a2t[row];
		const int32_t q0 = ioff[node], q1 = ioff[node + 1];
		const int64_t total = (int64_t)(q1 - q0) * npe;
		if (total > kCand) {
			if (lane == 0) atomicExch(err, 1);
			continue;
		}
		const int k = (int)total;
		for (int t = lane; t < k; t += 32) {
			const int32_t e = inc[q0 + t / npe];
			c[t] = t2a[ien[(int64_t)e * npe + t % npe]];
		}
		__syncwarp();
		for (int t = lane; t < k; t += 32) {
			const int32_t v = c[t];
			bool f = v >= 0;
			for (int j = 0; j < t && f; ++j) f = c[j] != v;
			fl[t] = f;
		}
		__syncwarp();
		if (!FILL) {
			int m = 0;
			for (int t = lane; t < k; t += 32) m += fl[t];
#pragma unroll
			for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
			if (lane == 0) cnt[row] = m;
		} else {
			const int32_t base = rp[row];
			for (int t = lane; t < k; t += 32) {
				if (!fl[t]) continue;
				const int32_t v = c[t];
				int rank = 0;
				for (int j = 0; j < k; ++j) rank += fl[j] && c[j] < v;
				col[base + rank] = v;
			}
		}
		__syncwarp();
	}
}

}  // namespace

// The DOF map on the device; fills h->t2a (device) and the host copies h_t2a, h_a2t, h_ctag, h->n.
int device_dofmap(rsd_ctx* ctx, rsd_heat* h) {
	const rsd_mesh* m = h->m;
	const int64_t nn = m->nnodes, ne = m->nelem;
	const int nf = m->nfaces;
	FaceTable ft{};
	for (int f = 0; f < nf; ++f) {
		int tmp[64];
		ft.count = face_nodes(m->nsd, m->order, f, tmp);
		if (ft.count > 16) return set_error(RSD_EINVAL, "faces with more than 16 nodes");
		for (int a = 0; a < ft.count; ++a) ft.node[f][a] = tmp[a];
	}
	const int nEss = (int)h->essTags.size();
	int32_t *rng = nullptr, *ess = nullptr, *isFree = nullptr, *scan = nullptr, *ctag = nullptr, *a2t = nullptr;
	uint32_t* win = nullptr;
	auto run = [&]() -> int {
		RSD_CUDA(cudaMalloc(&rng, sizeof(int32_t) * std::max<int64_t>(ne * nf, 1)));
		RSD_CUDA(cudaMalloc(&ess, sizeof(int32_t) * std::max(nEss, 1)));
		RSD_CUDA(cudaMalloc(&win, sizeof(uint32_t) * nn));
		RSD_CUDA(cudaMalloc(&isFree, sizeof(int32_t) * nn));
		RSD_CUDA(cudaMalloc(&scan, sizeof(int32_t) * (nn + 1)));
		RSD_CUDA(cudaMalloc(&ctag, sizeof(int32_t) * nn));
		RSD_CUDA(cudaMalloc(&a2t, sizeof(int32_t) * nn));
		RSD_CUDA(cudaMemcpyAsync(rng, m->h_rng.data(), sizeof(int32_t) * ne * nf, cudaMemcpyHostToDevice, ctx->stream));
		if (nEss) RSD_CUDA(cudaMemcpyAsync(ess, h->essTags.data(), sizeof(int32_t) * nEss, cudaMemcpyHostToDevice, ctx->stream));
		RSD_CUDA(cudaMemsetAsync(win, 0, sizeof(uint32_t) * nn, ctx->stream));
		k_mark_constrained<<<vec_grid(ctx, ne * nf), 256, 0, ctx->stream>>>(ne, nf, m->npe, rng, m->ien, ess, nEss, ft, win);
		k_dof_flags<<<vec_grid(ctx, nn), 256, 0, ctx->stream>>>(nn, win, rng, ess, nEss, isFree, ctag);
		RSD_CUDA(cudaGetLastError());
		int64_t n = 0;
		RSD_CHECK(exclusive_scan(ctx, isFree, scan, nn, &n));
		k_dof_number<<<vec_grid(ctx, nn), 256, 0, ctx->stream>>>(nn, isFree, scan, h->t2a, a2t);
		RSD_CUDA(cudaGetLastError());
		h->n = n;
		h->h_t2a.resize(nn);
		h->h_ctag.resize(nn);
		h->h_a2t.resize(n);
		RSD_CUDA(cudaMemcpyAsync(h->h_t2a.data(), h->t2a, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaMemcpyAsync(h->h_ctag.data(), ctag, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost, ctx->stream));
		if (n) RSD_CUDA(cudaMemcpyAsync(h->h_a2t.data(), a2t, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		return RSD_OK;
	};
	const int rc = run();
	cudaFree(rng); cudaFree(ess); cudaFree(win); cudaFree(isFree); cudaFree(scan); cudaFree(ctag); cudaFree(a2t);
	return rc;
}

// The CSR pattern on the device into host vectors rp (n + 1) and col; *fallback is set (and nothing
// else) when a row gathers more candidates than the warp buffer holds.
int device_pattern(rsd_ctx* ctx, const rsd_heat* h, std::vector<int32_t>& rp, std::vector<int32_t>& col, bool* fallback) {
	const rsd_mesh* m = h->m;
	const int64_t nn = m->nnodes, ne = m->nelem, n = h->n, tot = ne * m->npe;
	*fallback = false;
	int32_t *cnt = nullptr, *ioff = nullptr, *inc = nullptr, *a2t = nullptr, *rcnt = nullptr, *drp = nullptr, *dcol = nullptr, *err = nullptr;
	auto run = [&]() -> int {
		RSD_CUDA(cudaMalloc(&cnt, sizeof(int32_t) * nn));
		RSD_CUDA(cudaMalloc(&ioff, sizeof(int32_t) * (nn + 1)));
		RSD_CUDA(cudaMalloc(&inc, sizeof(int32_t) * std::max<int64_t>(tot, 1)));
		RSD_CUDA(cudaMalloc(&a2t, sizeof(int32_t) * std::max<int64_t>(n, 1)));
		RSD_CUDA(cudaMalloc(&rcnt, sizeof(int32_t) * std::max<int64_t>(n, 1)));
		RSD_CUDA(cudaMalloc(&drp, sizeof(int32_t) * (n + 1)));
		RSD_CUDA(cudaMalloc(&err, sizeof(int32_t)));
		RSD_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * nn, ctx->stream));
		RSD_CUDA(cudaMemsetAsync(err, 0, sizeof(int32_t), ctx->stream));
		if (n) RSD_CUDA(cudaMemcpyAsync(a2t, h->h_a2t.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, ctx->stream));
		k_incidence_count<<<vec_grid(ctx, tot), 256, 0, ctx->stream>>>(tot, m->ien, cnt);
		RSD_CUDA(cudaGetLastError());
		int64_t total = 0;
		RSD_CHECK(exclusive_scan(ctx, cnt, ioff, nn, &total));
		RSD_CUDA(cudaMemcpyAsync(cnt, ioff, sizeof(int32_t) * nn, cudaMemcpyDeviceToDevice, ctx->stream));   // cursors
		k_incidence_fill<<<vec_grid(ctx, tot), 256, 0, ctx->stream>>>(tot, m->npe, m->ien, cnt, inc);
		const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kRowWarpsSetup - 1) / kRowWarpsSetup, (int64_t)ctx->num_sms * 64));
		if (n) k_row_columns<false><<<blocks, 32 * kRowWarpsSetup, 0, ctx->stream>>>(n, m->npe, a2t, ioff, inc, m->ien, h->t2a, rcnt, nullptr, nullptr, err);
		RSD_CUDA(cudaGetLastError());
		int32_t herr = 0;
		RSD_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		if (herr) { *fallback = true; return RSD_OK; }
		int64_t nnz = 0;
		RSD_CHECK(exclusive_scan(ctx, rcnt, drp, n, &nnz));
		RSD_CUDA(cudaMalloc(&dcol, sizeof(int32_t) * std::max<int64_t>(nnz, 1)));
		if (n) k_row_columns<true><<<blocks, 32 * kRowWarpsSetup, 0, ctx->stream>>>(n, m->npe, a2t, ioff, inc, m->ien, h->t2a, nullptr, drp, dcol, err);
		RSD_CUDA(cudaGetLastError());
		rp.resize(n + 1);
		col.resize(nnz);
		RSD_CUDA(cudaMemcpyAsync(rp.data(), drp, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, ctx->stream));
		if (nnz) RSD_CUDA(cudaMemcpyAsync(col.data(), dcol, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, ctx->stream));
		RSD_CUDA(cudaStreamSynchronize(ctx->stream));
		return RSD_OK;
	};
	const int rc = run();
	cudaFree(cnt); cudaFree(ioff); cudaFree(inc); cudaFree(a2t); cudaFree(rcnt); cudaFree(drp); cudaFree(dcol); cudaFree(err);
	return rc;
}

}  // namespace rsd
