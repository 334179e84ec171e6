// Runtime part of the hpcscan_b200 C ABI: device selection, errors, memory, box copies,
// and the per-device scratch buffers used by reductions and table uploads.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "b200_common.cuh"

namespace b200 {

static thread_local char g_last_error[1024] = "";

int set_error(int code, const char* fmt, ...)
{
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
	va_end(ap);
	return code;
}

int cuda_error(cudaError_t err, const char* what)
{
	if (err == cudaSuccess) return B200_OK;
	int code = (err == cudaErrorMemoryAllocation) ? B200_ERR_NOMEM : B200_ERR_CUDA;
	return set_error(code, "%s: %s (%s)", what, cudaGetErrorString(err), cudaGetErrorName(err));
}

int check_launch(const char* what) { return cuda_error(cudaGetLastError(), what); }

// ---- per-device state -----------------------------------------------------------------------
namespace {
constexpr int kMaxDevices = 64;
struct DeviceState {
	void* scratch = nullptr;
	size_t scratch_bytes = 0;
	void* staging = nullptr;
	size_t staging_bytes = 0;
	int sms = 0;
};
DeviceState g_dev[kMaxDevices];
std::mutex g_mutex;

int current_device(int* dev)
{
	int rc = cuda_error(cudaGetDevice(dev), "cudaGetDevice");
	if (rc) return rc;
	if (*dev < 0 || *dev >= kMaxDevices) return set_error(B200_ERR_ARG, "device index %d", *dev);
	return B200_OK;
}
}  // namespace

int scratch(size_t bytes, void** ptr)
{
	int dev;
	if (int rc = current_device(&dev)) return rc;
	std::lock_guard<std::mutex> lock(g_mutex);
	DeviceState& s = g_dev[dev];
	if (s.scratch_bytes < bytes) {
		if (s.scratch) {
			// the old buffer may still be read by enqueued work
			cudaDeviceSynchronize();
			cudaFree(s.scratch);
			s.scratch = nullptr;
			s.scratch_bytes = 0;
		}
		size_t want = bytes < (1u << 20) ? (1u << 20) : bytes;
		if (int rc = cuda_error(cudaMalloc(&s.scratch, want), "cudaMalloc(scratch)")) return rc;
		s.scratch_bytes = want;
	}
	*ptr = s.scratch;
	return B200_OK;
}

int host_staging(size_t bytes, void** ptr)
{
	int dev;
	if (int rc = current_device(&dev)) return rc;
	std::lock_guard<std::mutex> lock(g_mutex);
	DeviceState& s = g_dev[dev];
	if (s.staging_bytes < bytes) {
		if (s.staging) {
			cudaDeviceSynchronize();
			cudaFreeHost(s.staging);
			s.staging = nullptr;
			s.staging_bytes = 0;
		}
		size_t want = bytes < 4096 ? 4096 : bytes;
		if (int rc = cuda_error(cudaMallocHost(&s.staging, want), "cudaMallocHost(staging)"))
			return rc;
		s.staging_bytes = want;
	}
	*ptr = s.staging;
	return B200_OK;
}

// The library's device-side error word (set by kernels that give up a bounded wait).
__device__ unsigned int g_device_error;

int device_error_word(unsigned int** ptr)
{
	int dev;
	if (int rc = current_device(&dev)) return rc;
	static unsigned int* cached[kMaxDevices] = {};
	if (!cached[dev]) {
		void* p = nullptr;
		if (int rc = cuda_error(cudaGetSymbolAddress(&p, g_device_error), "cudaGetSymbolAddress"))
			return rc;
		cached[dev] = static_cast<unsigned int*>(p);
	}
	*ptr = cached[dev];
	return B200_OK;
}

int num_sms()
{
	int dev = 0;
	if (current_device(&dev)) return 148;
	if (g_dev[dev].sms == 0) {
		int n = 0;
		cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
		g_dev[dev].sms = n > 0 ? n : 148;
	}
	return g_dev[dev].sms;
}

// ---- validation ---------------------------------------------------------------------------------
int check_layout(const b200_layout* lay)
{
	if (!lay) return set_error(B200_ERR_ARG, "layout is NULL");
	if (lay->dim < 1 || lay->dim > 3) return set_error(B200_ERR_ARG, "dim %d", lay->dim);
	if (lay->n1 < 1 || lay->n2 < 1 || lay->n3 < 1)
		return set_error(B200_ERR_ARG, "array dims %lld %lld %lld", (long long)lay->n1,
				(long long)lay->n2, (long long)lay->n3);
	if (lay->halo < 0 || lay->halo > 8) return set_error(B200_ERR_ARG, "halo %d", lay->halo);
	const int64_t s[3] = {lay->s1, lay->s2, lay->s3}, e[3] = {lay->e1, lay->e2, lay->e3};
	const int64_t n[3] = {lay->n1, lay->n2, lay->n3};
	for (int a = 0; a < 3; a++) {
		if (a < lay->dim) {
			if (s[a] - lay->halo < 0 || e[a] + lay->halo >= n[a] || e[a] < s[a])
				return set_error(B200_ERR_ARG,
						"axis %d: inner [%lld,%lld] with halo %d does not fit in %lld points", a + 1,
						(long long)s[a], (long long)e[a], lay->halo, (long long)n[a]);
		} else if (s[a] != 0 || e[a] != 0 || n[a] != 1) {
			return set_error(B200_ERR_ARG, "axis %d beyond dim must have n=1, s=e=0", a + 1);
		}
	}
	return B200_OK;
}

int check_box(const b200_layout* lay, const b200_box* b)
{
	if (!b) return set_error(B200_ERR_ARG, "box is NULL");
	if (b->i1s < 0 || b->i1e >= lay->n1 || b->i2s < 0 || b->i2e >= lay->n2 || b->i3s < 0 ||
			b->i3e >= lay->n3)
		return set_error(B200_ERR_ARG, "box [%lld,%lld]x[%lld,%lld]x[%lld,%lld] outside the array",
				(long long)b->i1s, (long long)b->i1e, (long long)b->i2s, (long long)b->i2e,
				(long long)b->i3s, (long long)b->i3e);
	// an end before its start would give negative extents, which the row walks would turn into
	// indices past the box
	if (b->i1e < b->i1s || b->i2e < b->i2s || b->i3e < b->i3s)
		return set_error(B200_ERR_ARG, "box [%lld,%lld]x[%lld,%lld]x[%lld,%lld] has an end before its start",
				(long long)b->i1s, (long long)b->i1e, (long long)b->i2s, (long long)b->i2e,
				(long long)b->i3s, (long long)b->i3e);
	return B200_OK;
}

int check_order(int order)
{
	if (order < 2 || order > 16 || (order & 1))
		return set_error(B200_ERR_ARG, "FD order %d not supported (2..16, even)", order);
	return B200_OK;
}

int check_field(const b200_field& f, const char* name)
{
	if (!f.data) return set_error(B200_ERR_ARG, "field %s: NULL data", name);
	if (dtype_size(f.dtype) == 0) return set_error(B200_ERR_ARG, "field %s: dtype %d", name, f.dtype);
	if (!(f.scale > 0.0f)) return set_error(B200_ERR_ARG, "field %s: scale must be > 0", name);
	return B200_OK;
}

}  // namespace b200

using namespace b200;

extern "C" {

const char* b200_last_error(void) { return g_last_error; }

int b200_device_count(int* count)
{
	if (!count) return set_error(B200_ERR_ARG, "count is NULL");
	return cuda_error(cudaGetDeviceCount(count), "cudaGetDeviceCount");
}

int b200_init(int device)
{
	int n = 0;
	if (int rc = cuda_error(cudaGetDeviceCount(&n), "cudaGetDeviceCount")) return rc;
	if (n <= 0) return set_error(B200_ERR_CUDA, "no CUDA device");
	if (device < 0) device = 0;
	device %= n;
	if (int rc = cuda_error(cudaSetDevice(device), "cudaSetDevice")) return rc;
	cudaDeviceProp prop;
	if (int rc = cuda_error(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties"))
		return rc;
	if (prop.major < 10)
		return set_error(B200_ERR_UNSUPPORTED, "device %d (%s) is sm_%d%d; this build targets sm_100a",
				device, prop.name, prop.major, prop.minor);
	cudaFree(nullptr);   // create the context now
	return B200_OK;
}

int b200_malloc(void** dptr, size_t bytes)
{
	if (!dptr) return set_error(B200_ERR_ARG, "dptr is NULL");
	*dptr = nullptr;
	if (bytes == 0) return B200_OK;
	return cuda_error(cudaMalloc(dptr, bytes), "cudaMalloc");
}

int b200_free(void* dptr)
{
	if (!dptr) return B200_OK;
	return cuda_error(cudaFree(dptr), "cudaFree");
}

int b200_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream)
{
	if (bytes == 0) return B200_OK;
	if (!dst || !src) return set_error(B200_ERR_ARG, "NULL pointer");
	return cuda_error(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream)),
			"cudaMemcpyAsync(H2D)");
}

int b200_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream)
{
	if (bytes == 0) return B200_OK;
	if (!dst || !src) return set_error(B200_ERR_ARG, "NULL pointer");
	int rc = cuda_error(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)),
			"cudaMemcpyAsync(D2H)");
	if (rc) return rc;
	return cuda_error(cudaStreamSynchronize(as_stream(stream)), "cudaStreamSynchronize");
}

int b200_memcpy_d2d(void* dst, const void* src, size_t bytes, void* stream)
{
	if (bytes == 0) return B200_OK;
	if (!dst || !src) return set_error(B200_ERR_ARG, "NULL pointer");
	return cuda_error(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)),
			"cudaMemcpyAsync(D2D)");
}

int b200_memset(void* dptr, int value, size_t bytes, void* stream)
{
	if (bytes == 0) return B200_OK;
	if (!dptr) return set_error(B200_ERR_ARG, "NULL pointer");
	return cuda_error(cudaMemsetAsync(dptr, value, bytes, as_stream(stream)), "cudaMemsetAsync");
}

int b200_device_status(int* status, int clear)
{
	if (!status) return set_error(B200_ERR_ARG, "status is NULL");
	unsigned int v = 0;
	int rc = cuda_error(cudaMemcpyFromSymbol(&v, g_device_error, sizeof(v)), "cudaMemcpyFromSymbol");
	if (rc) return rc;
	*status = (int)v;
	if (clear && v) {
		const unsigned int zero = 0;
		rc = cuda_error(cudaMemcpyToSymbol(g_device_error, &zero, sizeof(zero)), "cudaMemcpyToSymbol");
	}
	return rc;
}

int b200_stream_sync(void* stream)
{
	return cuda_error(cudaStreamSynchronize(as_stream(stream)), "cudaStreamSynchronize");
}

static int copy_box(const b200_layout* lay, int es, void* dst, const void* src,
		const b200_box* box, cudaMemcpyKind kind, void* stream)
{
	if (int rc = check_layout(lay)) return rc;
	if (int rc = check_box(lay, box)) return rc;
	if (es <= 0 || es > 8) return set_error(B200_ERR_ARG, "element size %d", es);
	if (!dst || !src) return set_error(B200_ERR_ARG, "NULL pointer");
	// one 3-D copy: rows of (i1e-i1s+1) elements, pitch n1, n2 rows per plane
	cudaMemcpy3DParms p = {};
	const size_t pitch = (size_t)lay->n1 * es;
	p.srcPtr = make_cudaPitchedPtr(const_cast<void*>(src), pitch, (size_t)lay->n1, (size_t)lay->n2);
	p.dstPtr = make_cudaPitchedPtr(dst, pitch, (size_t)lay->n1, (size_t)lay->n2);
	p.srcPos = make_cudaPos((size_t)box->i1s * es, (size_t)box->i2s, (size_t)box->i3s);
	p.dstPos = p.srcPos;
	p.extent = make_cudaExtent((size_t)(box->i1e - box->i1s + 1) * es,
			(size_t)(box->i2e - box->i2s + 1), (size_t)(box->i3e - box->i3s + 1));
	p.kind = kind;
	int rc = cuda_error(cudaMemcpy3DAsync(&p, as_stream(stream)), "cudaMemcpy3DAsync");
	if (rc) return rc;
	if (kind == cudaMemcpyDeviceToHost)
		return cuda_error(cudaStreamSynchronize(as_stream(stream)), "cudaStreamSynchronize");
	return B200_OK;
}

int b200_copy_box_d2h(const b200_layout* lay, int elem_size, void* host, const void* dev,
		const b200_box* box, void* stream)
{
	return copy_box(lay, elem_size, host, dev, box, cudaMemcpyDeviceToHost, stream);
}

int b200_copy_box_h2d(const b200_layout* lay, int elem_size, void* dev, const void* host,
		const b200_box* box, void* stream)
{
	return copy_box(lay, elem_size, dev, host, box, cudaMemcpyHostToDevice, stream);
}

}  // extern "C"
