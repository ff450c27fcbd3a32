// Binary containers in the reference's linalg::io format, for interop and
// for checkpoints of serving members.
//
// The reference writes each dense vector or matrix as (include/linalg/io.h:
// 66-94, 425-497): a 32-bit magic number (container | layout | value type:
// 'v','e' or 'm','a' in the high bytes, 'd' for dense, then 'd' or 's' for
// FP64 / FP32 values), three 32-bit ints (rows, cols, values), and the
// values, column-major (a matrix of n points in dims columns is the x[d*n+p]
// layout).  A sparse one ('s' layout; io.h:432-470, 497-532) has the three
// ints (rows, cols, nonzeros), then for a matrix its CSR row starts (rows + 1
// ints, none when rows is 0), the nonzeros' indices (ints) and their values.
// Scalars are their raw bytes.  Objects follow each other in one stream.
// Host byte order (little-endian on every supported host).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "ibk_internal.h"

namespace ibk {
namespace {

constexpr int kVector = 0x65760000, kMatrix = 0x616d0000, kDense = 0x6400, kSparse = 0x7300;
constexpr int kF64 = 0x64, kF32 = 0x73;

struct File {
	FILE* f = nullptr;
	~File() { if (f) std::fclose(f); }
};

ibk_status open_at(File& file, const char* path, const char* mode, long long offset)
{
	file.f = std::fopen(path, mode);
	if (!file.f) return set_error(IBK_ERR_INVALID_ARGUMENT, std::string("cannot open ") + path);
	if (offset > 0 && std::fseek(file.f, (long) offset, SEEK_SET) != 0)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "offset past the end of the file");
	return IBK_OK;
}

} // namespace
} // namespace ibk

using namespace ibk;

extern "C" {

ibk_status ibk_io_write_dense(const char* path, int append, int matrix, int rows, int cols, const double* values)
{
	if (!path || rows < 0 || cols < 0 || (!matrix && cols != 1) || (rows > 0 && cols > 0 && !values))
		return set_error(IBK_ERR_INVALID_ARGUMENT, "bad path, shape or values");
	const long long count = (long long) rows * cols;
	if (count > 0x7fffffffLL) return set_error(IBK_ERR_INVALID_ARGUMENT, "object too large for 32-bit counts");
	File file;
	ibk_status st = open_at(file, path, append ? "ab" : "wb", 0);
	if (st != IBK_OK) return st;
	const int head[4] = {(matrix ? kMatrix : kVector) | kDense | kF64, rows, cols, (int) count};
	if (std::fwrite(head, sizeof(int), 4, file.f) != 4 ||
	    std::fwrite(values, sizeof(double), (size_t) count, file.f) != (size_t) count)
		return set_error(IBK_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
	return IBK_OK;
}

ibk_status ibk_io_write_scalar(const char* path, int append, double value)
{
	if (!path) return set_error(IBK_ERR_INVALID_ARGUMENT, "null path");
	File file;
	ibk_status st = open_at(file, path, append ? "ab" : "wb", 0);
	if (st != IBK_OK) return st;
	if (std::fwrite(&value, sizeof(double), 1, file.f) != 1)
		return set_error(IBK_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
	return IBK_OK;
}

ibk_status ibk_io_read_dense(const char* path, long long offset, ibk_io_header* header, double* values,
                             long long capacity, long long* next_offset)
{
	if (!path || !header || offset < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "bad path, header or offset");
	File file;
	ibk_status st = open_at(file, path, "rb", offset);
	if (st != IBK_OK) return st;
	int head[4];
	if (std::fread(head, sizeof(int), 4, file.f) != 4)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated header");
	const int container = head[0] & 0x7fff0000, layout = head[0] & 0xff00, type = head[0] & 0xff;
	if ((container != kVector && container != kMatrix) || (type != kF64 && type != kF32))
		return set_error(IBK_ERR_INVALID_ARGUMENT, "not a linalg::io container");
	if (layout != kDense) return set_error(IBK_ERR_INVALID_ARGUMENT, "a sparse container (ibk_io_read_sparse)");
	if (head[1] < 0 || head[2] < 0 || (long long) head[1] * head[2] != head[3])
		return set_error(IBK_ERR_INVALID_ARGUMENT, "inconsistent header");
	header->magic = head[0];
	header->matrix = container == kMatrix;
	header->rows = head[1];
	header->cols = head[2];
	header->count = head[3];
	const size_t width = type == kF64 ? sizeof(double) : sizeof(float);
	const long long data_end = offset + 16 + (long long) head[3] * (long long) width;
	if (values) {
		if (capacity < head[3]) return set_error(IBK_ERR_CAPACITY, "value buffer too small");
		if (type == kF64) {
			if (std::fread(values, sizeof(double), (size_t) head[3], file.f) != (size_t) head[3])
				return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated values");
		} else {
			std::vector<float> tmp((size_t) head[3]);
			if (std::fread(tmp.data(), sizeof(float), tmp.size(), file.f) != tmp.size())
				return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated values");
			for (size_t i = 0; i < tmp.size(); ++i) values[i] = tmp[i];
		}
	}
	if (next_offset) *next_offset = data_end;
	return IBK_OK;
}

ibk_status ibk_io_write_sparse(const char* path, int append, int matrix, int rows, int cols, int nonzeros,
                               const int* starts, const int* indices, const double* values)
{
	if (!path || rows < 0 || cols < 0 || nonzeros < 0 || (!matrix && cols != 1) ||
	    (matrix && rows > 0 && !starts) || (nonzeros > 0 && (!indices || !values)))
		return set_error(IBK_ERR_INVALID_ARGUMENT, "bad path, shape or arrays");
	File file;
	ibk_status st = open_at(file, path, append ? "ab" : "wb", 0);
	if (st != IBK_OK) return st;
	const int head[4] = {(matrix ? kMatrix : kVector) | kSparse | kF64, rows, cols, nonzeros};
	const size_t ns = matrix && rows > 0 ? (size_t) rows + 1 : 0;
	if (std::fwrite(head, sizeof(int), 4, file.f) != 4 || (ns && std::fwrite(starts, sizeof(int), ns, file.f) != ns) ||
	    std::fwrite(indices, sizeof(int), (size_t) nonzeros, file.f) != (size_t) nonzeros ||
	    std::fwrite(values, sizeof(double), (size_t) nonzeros, file.f) != (size_t) nonzeros)
		return set_error(IBK_ERR_INVALID_ARGUMENT, std::string("write failed: ") + path);
	return IBK_OK;
}

ibk_status ibk_io_read_sparse(const char* path, long long offset, ibk_io_header* header, int* starts,
                              int* indices, double* values, long long capacity, long long* next_offset)
{
	if (!path || !header || offset < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "bad path, header or offset");
	File file;
	ibk_status st = open_at(file, path, "rb", offset);
	if (st != IBK_OK) return st;
	int head[4];
	if (std::fread(head, sizeof(int), 4, file.f) != 4)
		return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated header");
	const int container = head[0] & 0x7fff0000, layout = head[0] & 0xff00, type = head[0] & 0xff;
	if ((container != kVector && container != kMatrix) || (type != kF64 && type != kF32))
		return set_error(IBK_ERR_INVALID_ARGUMENT, "not a linalg::io container");
	if (layout != kSparse) return set_error(IBK_ERR_INVALID_ARGUMENT, "not a sparse container");
	if (head[1] < 0 || head[2] < 0 || head[3] < 0 || (long long) head[3] > (long long) head[1] * head[2])
		return set_error(IBK_ERR_INVALID_ARGUMENT, "inconsistent header");
	header->magic = head[0];
	header->matrix = container == kMatrix;
	header->rows = head[1];
	header->cols = head[2];
	header->count = head[3];
	const long long ns = header->matrix && head[1] > 0 ? (long long) head[1] + 1 : 0;
	const size_t width = type == kF64 ? sizeof(double) : sizeof(float);
	const long long data_end = offset + 16 + 4 * ns + 4 * (long long) head[3] + (long long) head[3] * (long long) width;
	if (starts || indices || values) {
		if (!indices || !values || (ns && !starts)) return set_error(IBK_ERR_INVALID_ARGUMENT, "null output array");
		if (capacity < head[3]) return set_error(IBK_ERR_CAPACITY, "index / value buffers too small");
		if (ns && std::fread(starts, sizeof(int), (size_t) ns, file.f) != (size_t) ns)
			return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated row starts");
		if (std::fread(indices, sizeof(int), (size_t) head[3], file.f) != (size_t) head[3])
			return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated indices");
		if (type == kF64) {
			if (std::fread(values, sizeof(double), (size_t) head[3], file.f) != (size_t) head[3])
				return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated values");
		} else {
			std::vector<float> tmp((size_t) head[3]);
			if (std::fread(tmp.data(), sizeof(float), tmp.size(), file.f) != tmp.size())
				return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated values");
			for (size_t i = 0; i < tmp.size(); ++i) values[i] = tmp[i];
		}
	}
	if (next_offset) *next_offset = data_end;
	return IBK_OK;
}

ibk_status ibk_io_read_scalar(const char* path, long long offset, double* value, long long* next_offset)
{
	if (!path || !value || offset < 0) return set_error(IBK_ERR_INVALID_ARGUMENT, "bad path, value or offset");
	File file;
	ibk_status st = open_at(file, path, "rb", offset);
	if (st != IBK_OK) return st;
	if (std::fread(value, sizeof(double), 1, file.f) != 1) return set_error(IBK_ERR_INVALID_ARGUMENT, "truncated scalar");
	if (next_offset) *next_offset = offset + (long long) sizeof(double);
	return IBK_OK;
}

} // extern "C"
