// PMSH mesh input (the reference's binary mesh format, MeshIO::readBinary, src/io/MeshIO.cpp:84-151):
// a little-endian header (magic "PMSH", version 1, parametric and spatial dimension, element family,
// basis type, node and element counts, nodes and faces per element, the basis orders, an IGA flag and
// the extraction-operator size, all as MeshIO::writeBinary writes them) followed by xyz (FP64,
// node-major), ien (uint64, element-major) and rng (int32 per element face).  The reader fills host
// arrays; rsd_mesh_read_pmsh hands them to rsd_mesh_create.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "rsd_internal.cuh"

namespace rsd {
namespace {

constexpr uint32_t kPmshMagic = 0x504D5348u;   // "PMSH"
constexpr uint32_t kPmshVersion = 1u;

struct File {
	FILE* f = nullptr;
	~File() { if (f) std::fclose(f); }
};

// little-endian values of 1, 4 or 8 bytes, whatever the host's byte order
template <typename T>
bool read_le(FILE* f, T* out, size_t count = 1) {
	static_assert(sizeof(T) == 1 || sizeof(T) == 4 || sizeof(T) == 8, "1-, 4- or 8-byte values");
	if (count == 0) return true;
	if (std::fread(out, sizeof(T), count, f) != count) return false;
	const uint16_t probe = 1;
	if (*reinterpret_cast<const uint8_t*>(&probe) == 1 || sizeof(T) == 1) return true;
	for (size_t i = 0; i < count; ++i) {
		unsigned char* b = reinterpret_cast<unsigned char*>(out + i);
		for (size_t k = 0; k < sizeof(T) / 2; ++k) std::swap(b[k], b[sizeof(T) - 1 - k]);
	}
	return true;
}

int read_pmsh(const char* path, rsd_pmsh_info* info, std::vector<double>* xyz, std::vector<uint64_t>* ien, std::vector<int32_t>* rng) {
	File file;
	file.f = std::fopen(path, "rb");
	if (!file.f) return set_error(RSD_EINVAL, std::string("cannot open PMSH file '") + path + "'");
	FILE* f = file.f;
	uint32_t magic = 0, version = 0, hdr[8] = {}, norders = 0;
	if (!read_le(f, &magic) || magic != kPmshMagic) return set_error(RSD_EINVAL, "bad magic number: not a PMSH file");
	if (!read_le(f, &version) || version != kPmshVersion) return set_error(RSD_EINVAL, "unsupported PMSH version " + std::to_string(version));
	if (!read_le(f, hdr, 8) || !read_le(f, &norders)) return set_error(RSD_EINVAL, "unexpected end of file in the PMSH header");
	if (norders > 3) return set_error(RSD_EINVAL, "PMSH header lists more than 3 basis orders");
	uint32_t orders[3] = {0, 0, 0};
	uint8_t iga = 0;
	uint64_t csize = 0;
	if (!read_le(f, orders, norders) || !read_le(f, &iga) || !read_le(f, &csize)) return set_error(RSD_EINVAL, "unexpected end of file in the PMSH header");
	rsd_pmsh_info I{};
	I.parametric_dim = (int32_t)hdr[0];
	I.spatial_dim = (int32_t)hdr[1];
	I.family = (int32_t)hdr[2];
	I.basis = (int32_t)hdr[3];
	I.num_nodes = hdr[4];
	I.num_elements = hdr[5];
	I.nodes_per_element = (int32_t)hdr[6];
	I.faces_per_element = (int32_t)hdr[7];
	I.num_orders = (int32_t)norders;
	for (int i = 0; i < 3; ++i) I.order[i] = (int32_t)orders[i];
	I.iga = iga ? 1 : 0;
	if (I.spatial_dim < 1 || I.spatial_dim > 3 || I.parametric_dim < 1 || I.parametric_dim > 3)
		return set_error(RSD_EINVAL, "PMSH dimensions out of range");
	if (info) *info = I;
	if (!xyz && !ien && !rng) return RSD_OK;
	const uint64_t nx = (uint64_t)I.num_nodes * (uint64_t)I.spatial_dim;
	const uint64_t ni = (uint64_t)I.num_elements * (uint64_t)I.nodes_per_element;
	const uint64_t nr = (uint64_t)I.num_elements * (uint64_t)I.faces_per_element;
	std::vector<double> x(nx);
	std::vector<uint64_t> c(ni);
	std::vector<int32_t> r(nr);
	if (!read_le(f, x.data(), x.size()) || !read_le(f, c.data(), c.size()) || !read_le(f, r.data(), r.size()))
		return set_error(RSD_EINVAL, "unexpected end of file in the PMSH data");
	for (uint64_t v : c)
		if (v >= (uint64_t)I.num_nodes) return set_error(RSD_EINVAL, "PMSH connectivity references a missing node");
	if (xyz) *xyz = std::move(x);
	if (ien) *ien = std::move(c);
	if (rng) *rng = std::move(r);
	return RSD_OK;
}

}  // namespace
}  // namespace rsd

using namespace rsd;

extern "C" {

int rsd_pmsh_read(const char* path, rsd_pmsh_info* info, double* xyz, int64_t* ien, int32_t* rng) {
	if (!path) return set_error(RSD_EINVAL, "null path");
	rsd_pmsh_info I{};
	if (!xyz && !ien && !rng) return read_pmsh(path, info, nullptr, nullptr, nullptr);
	std::vector<double> x;
	std::vector<uint64_t> c;
	std::vector<int32_t> r;
	RSD_CHECK(read_pmsh(path, &I, &x, &c, &r));
	if (info) *info = I;
	if (xyz) std::memcpy(xyz, x.data(), sizeof(double) * x.size());
	if (ien) for (size_t i = 0; i < c.size(); ++i) ien[i] = (int64_t)c[i];
	if (rng) std::memcpy(rng, r.data(), sizeof(int32_t) * r.size());
	return RSD_OK;
}

int rsd_mesh_read_pmsh(rsd_ctx* ctx, const char* path, rsd_mesh** out) {
	if (!ctx || !path || !out) return set_error(RSD_EINVAL, "null argument");
	rsd_pmsh_info I{};
	std::vector<double> x;
	std::vector<uint64_t> c;
	std::vector<int32_t> r;
	RSD_CHECK(read_pmsh(path, &I, &x, &c, &r));
	// the Lagrange quad/hex meshes of equal order in every direction the device path takes
	const bool quad = I.family == 0 && I.parametric_dim == 2, hex = I.family == 2 && I.parametric_dim == 3;
	if (!quad && !hex) return set_error(RSD_EINVAL, "PMSH element family: quadrilaterals or hexahedra only");
	if (I.basis != 0 || I.iga) return set_error(RSD_EINVAL, "PMSH basis: Lagrange (FEM) only");
	if (I.spatial_dim != I.parametric_dim) return set_error(RSD_EINVAL, "PMSH meshes embedded in a higher dimension are not supported");
	if (I.num_orders != I.parametric_dim) return set_error(RSD_EINVAL, "PMSH header: one basis order per parametric direction");
	for (int i = 1; i < I.num_orders; ++i)
		if (I.order[i] != I.order[0]) return set_error(RSD_EINVAL, "PMSH basis orders must be equal in every direction");
	const int p = I.order[0];
	const int npe = (p + 1) * (p + 1) * (hex ? p + 1 : 1);
	if (I.nodes_per_element != npe || I.faces_per_element != 2 * I.parametric_dim)
		return set_error(RSD_EINVAL, "PMSH nodes or faces per element do not match the element type");
	std::vector<int64_t> ien(c.begin(), c.end());
	return rsd_mesh_create(ctx, I.spatial_dim, p, I.num_nodes, I.num_elements, x.data(), ien.data(), r.data(), out);
}

}  // extern "C"
