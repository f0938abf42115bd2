#include "rqc_runtime.h"

#include <stdio.h>
#include <map>

namespace rqc {

static std::map<int, Runtime*> g_runtimes;
static int g_last_error = 0;

Runtime* runtime()
{
	int dev = -1;
	if (cudaGetDevice(&dev) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "rqcopt_gpu: no CUDA device available\n");
		return nullptr;
	}
	auto it = g_runtimes.find(dev);
	if (it != g_runtimes.end()) return it->second;
	Runtime* rt = new Runtime();
	rt->device = dev;
	if (cudaDeviceGetAttribute(&rt->num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
	    cudaStreamCreateWithFlags(&rt->stream, cudaStreamNonBlocking) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "rqcopt_gpu: initialising device %d failed\n", dev);
		delete rt;
		return nullptr;
	}
	g_runtimes[dev] = rt;
	return rt;
}

int cuda_check(cudaError_t e, const char* what, const char* file, int line)
{
	if (e == cudaSuccess) return OK;
	fprintf(stderr, "rqcopt_gpu: CUDA error '%s' in %s (%s:%d)\n", cudaGetErrorString(e), what, file, line);
	return E_CUDA;
}

void set_last_error(int code) { g_last_error = code; }
int take_last_error() { int e = g_last_error; g_last_error = 0; return e; }

void fail_arg(const char* fn, const char* msg)
{
	fprintf(stderr, "rqcopt_gpu: %s: %s\n", fn, msg);
	set_last_error(E_ARG);
}

int ensure_device(Buffer& b, size_t bytes)
{
	if (b.bytes >= bytes && b.ptr) return OK;
	if (b.ptr) {
		cudaFree(b.ptr);
		b.ptr = nullptr;
		b.bytes = 0;
	}
	if (bytes == 0) return OK;
	if (cudaMalloc(&b.ptr, bytes) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "rqcopt_gpu: allocating %zu bytes of device memory failed\n", bytes);
		b.ptr = nullptr;
		return E_ALLOC;
	}
	b.bytes = bytes;
	return OK;
}

int ensure_host_pinned(Buffer& b, size_t bytes)
{
	if (b.bytes >= bytes && b.ptr) return OK;
	if (b.ptr) {
		cudaFreeHost(b.ptr);
		b.ptr = nullptr;
		b.bytes = 0;
	}
	if (bytes == 0) return OK;
	if (cudaMallocHost(&b.ptr, bytes) != cudaSuccess) {
		cudaGetLastError();
		fprintf(stderr, "rqcopt_gpu: allocating %zu bytes of pinned host memory failed\n", bytes);
		b.ptr = nullptr;
		return E_ALLOC;
	}
	b.bytes = bytes;
	return OK;
}

bool is_device_pointer(const void* p)
{
	cudaPointerAttributes a;
	if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		return false;
	}
	return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

int span_in(Runtime& rt, const void* p, size_t bytes, int slot, DeviceSpan& s)
{
	s.bytes = bytes;
	if (is_device_pointer(p)) {
		s.dev = const_cast<void*>(p);
		s.host = nullptr;
		return OK;
	}
	int ret = ensure_device(rt.stage[slot], bytes);
	if (ret) return ret;
	s.dev = rt.stage[slot].ptr;
	s.host = const_cast<void*>(p);
	return RQC_CUDA(cudaMemcpyAsync(s.dev, p, bytes, cudaMemcpyHostToDevice, rt.stream));
}

int span_out(Runtime& rt, void* p, size_t bytes, int slot, DeviceSpan& s)
{
	s.bytes = bytes;
	if (is_device_pointer(p)) {
		s.dev = p;
		s.host = nullptr;
		return OK;
	}
	int ret = ensure_device(rt.stage[slot], bytes);
	if (ret) return ret;
	s.dev = rt.stage[slot].ptr;
	s.host = p;
	return OK;
}

int span_finish(Runtime& rt, DeviceSpan& s)
{
	if (!s.host) return OK;
	return RQC_CUDA(cudaMemcpyAsync(s.host, s.dev, s.bytes, cudaMemcpyDeviceToHost, rt.stream));
}

static cudaEvent_t take_event(Runtime& rt)
{
	if (!rt.event_pool.empty()) {
		cudaEvent_t e = rt.event_pool.back();
		rt.event_pool.pop_back();
		return e;
	}
	cudaEvent_t e;
	cudaEventCreate(&e);
	return e;
}

int sync(Runtime& rt)
{
	int ret = RQC_CUDA(cudaStreamSynchronize(rt.stream));
	for (auto& p : rt.pending) {
		float ms = 0;
		if (ret == OK && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
			rt.time_ms[p.cls] += ms;
			rt.time_count[p.cls] += 1;
		}
		rt.event_pool.push_back(p.a);
		rt.event_pool.push_back(p.b);
	}
	rt.pending.clear();
	return ret;
}

void launch_begin(Runtime& rt, int cls, cudaEvent_t* ev_start)
{
	rt.launches++;
	*ev_start = nullptr;
	if (rt.timing) {
		*ev_start = take_event(rt);
		cudaEventRecord(*ev_start, rt.stream);
	}
	(void)cls;
}

void launch_end(Runtime& rt, int cls, cudaEvent_t ev_start)
{
	if (ev_start) {
		cudaEvent_t b = take_event(rt);
		cudaEventRecord(b, rt.stream);
		rt.pending.push_back({ev_start, b, cls});
		if (rt.pending.size() > 4096) sync(rt);
	}
}

}  // namespace rqc
