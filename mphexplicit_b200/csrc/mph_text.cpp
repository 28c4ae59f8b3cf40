// mph_text.cpp — host side of the device text writers: document assembly,
// the writer thread, and mph_format_e.
#include "mph_text.h"

#include <cstdio>
#include <cstring>
#include <vector>

#include "mph_b200.h"

namespace mph {

bool text_add(TextDoc& d, const char* head, int kind, int n, const void* src0, const void* src1, const void* src2) {
    const int len = head ? (int)std::strlen(head) : 0;
    if (d.nsec >= kTextMaxSections || len > kTextMaxUnit || d.head_used + len > kTextHeadPool || n < 0 ||
        kind < 0 || kind >= kRecKinds)
        return false;
    TextSection& s = d.sec[d.nsec++];
    s.kind = kind;
    s.n = kind == kRecNone ? 0 : n;
    s.head_off = d.head_used;
    s.head_len = len;
    s.first_block = 0;
    s.src0 = src0;
    s.src1 = src1;
    s.src2 = src2;
    if (len) std::memcpy(d.head + d.head_used, head, (size_t)len);
    d.head_used += len;
    return true;
}

TextWriter::TextWriter(int device) : device_(device) {
    th_ = std::thread([this] { run(); });
}

TextWriter::~TextWriter() {
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    if (th_.joinable()) th_.join();
    for (Slot& s : slot_) {
        cudaFree(s.text);
        cudaFree(s.blk);
        cudaFree(s.unit_len);
        cudaFree(s.off);
        if (s.done) cudaEventDestroy(s.done);
    }
    if (pinned_) cudaFreeHost(pinned_);
    if (total_) cudaFreeHost(total_);
    if (copy_) cudaStreamDestroy(copy_);
}

void TextWriter::fail(int code, const std::string& msg) {
    std::lock_guard<std::mutex> g(mu_);
    if (err_code_ == 0) {
        err_code_ = code;
        err_msg_ = msg;
    }
}

#define TW_CUDA(call, what)                                                                  \
    do {                                                                                     \
        const cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                             \
            if (err) *err = std::string(what) + ": " + cudaGetErrorString(e_);               \
            return MPH_ERR_CUDA;                                                             \
        }                                                                                    \
    } while (0)

int TextWriter::submit(TextDoc& doc, cudaStream_t stream, const std::string& path, std::string* err, int* launches) {
    const int nblocks = text_blocks(doc);
    const size_t need = text_max_bytes(doc);
    int k;
    {
        std::unique_lock<std::mutex> g(mu_);
        k = next_;
        cv_.wait(g, [&] { return !slot_[k].busy; });  // its previous document has been copied out
        next_ ^= 1;
    }
    Slot& s = slot_[k];
    if (!s.done) TW_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming), "cudaEventCreate");
    if (s.cap < need) {
        cudaFree(s.text);
        s.text = nullptr;
        s.cap = 0;
        TW_CUDA(cudaMalloc(&s.text, need + (need >> 3) + 256), "cudaMalloc(text)");
        s.cap = need + (need >> 3) + 256;
    }
    if (s.blk_cap < nblocks) {
        cudaFree(s.blk);
        cudaFree(s.unit_len);
        cudaFree(s.off);
        s.blk = nullptr;
        s.unit_len = nullptr;
        s.off = nullptr;
        s.blk_cap = 0;
        TW_CUDA(cudaMalloc(&s.blk, (size_t)nblocks * sizeof(uint32_t)), "cudaMalloc(text blocks)");
        TW_CUDA(cudaMalloc(&s.unit_len, (size_t)nblocks * kTextBlockUnits * sizeof(uint16_t)), "cudaMalloc(text lengths)");
        TW_CUDA(cudaMalloc(&s.off, ((size_t)nblocks + 2) * sizeof(unsigned long long)), "cudaMalloc(text offsets)");
        s.blk_cap = nblocks;
    }
    const int nl = launch_text(doc, s.unit_len, s.blk, s.off, s.text, stream);
    if (launches) *launches = nl;
    TW_CUDA(cudaGetLastError(), "text kernels");
    TW_CUDA(cudaEventRecord(s.done, stream), "cudaEventRecord");
    {
        std::lock_guard<std::mutex> g(mu_);
        s.busy = true;
        q_.push_back(Job{k, nblocks, path});
        ++inflight_;
    }
    cv_.notify_all();
    return MPH_OK;
}

int TextWriter::wait(std::string* err) {
    std::unique_lock<std::mutex> g(mu_);
    cv_.wait(g, [&] { return inflight_ == 0; });
    const int code = err_code_;
    if (code != 0 && err) *err = err_msg_;
    err_code_ = 0;
    err_msg_.clear();
    return code;
}

void TextWriter::run() {
    cudaSetDevice(device_);
    bool ready = cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking) == cudaSuccess &&
                 cudaHostAlloc(&total_, 2 * sizeof(unsigned long long), cudaHostAllocDefault) == cudaSuccess;
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> g(mu_);
            cv_.wait(g, [&] { return stop_ || !q_.empty(); });
            if (q_.empty()) return;  // stop_ with nothing left to write
            job = q_.front();
            q_.pop_front();
        }
        Slot& s = slot_[job.slot];
        size_t bytes = 0;
        bool ok = ready;
        if (!ready) fail(MPH_ERR_CUDA, "text writer: stream set-up failed");
        // the document's bytes: count, then the text itself
        if (ok && (cudaStreamWaitEvent(copy_, s.done, 0) != cudaSuccess ||
                   cudaMemcpyAsync(total_, s.off + job.nblocks, 2 * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, copy_) != cudaSuccess ||
                   cudaStreamSynchronize(copy_) != cudaSuccess)) {
            ok = false;
            fail(MPH_ERR_CUDA, std::string("text writer: ") + cudaGetErrorString(cudaGetLastError()));
        }
        if (ok) {
            bytes = (size_t)total_[0];
            if (bytes > s.cap || total_[1] != 0) {
                ok = false;
                fail(MPH_ERR_DEVICE, "text writer: a record's text did not have its counted length");
            }
        }
        if (ok && bytes > pinned_cap_) {
            if (pinned_) cudaFreeHost(pinned_);
            pinned_ = nullptr;
            pinned_cap_ = 0;
            if (cudaHostAlloc(&pinned_, bytes + (bytes >> 3), cudaHostAllocDefault) != cudaSuccess) {
                ok = false;
                fail(MPH_ERR_NOMEM, "text writer: pinned host buffer");
            } else {
                pinned_cap_ = bytes + (bytes >> 3);
            }
        }
        if (ok && bytes > 0 &&
            (cudaMemcpyAsync(pinned_, s.text, bytes, cudaMemcpyDeviceToHost, copy_) != cudaSuccess ||
             cudaStreamSynchronize(copy_) != cudaSuccess)) {
            ok = false;
            fail(MPH_ERR_CUDA, std::string("text writer: ") + cudaGetErrorString(cudaGetLastError()));
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            s.busy = false;  // the slot may be formatted into again
        }
        cv_.notify_all();
        if (ok) {
            FILE* fp = std::fopen(job.path.c_str(), "w");
            if (!fp) {
                fail(MPH_ERR_IO, "cannot write " + job.path);
            } else {
                const bool wrote = std::fwrite(pinned_, 1, bytes, fp) == bytes;
                const bool closed = std::fclose(fp) == 0;
                if (!wrote || !closed) fail(MPH_ERR_IO, "cannot write " + job.path);
            }
        }
        {
            std::lock_guard<std::mutex> g(mu_);
            --inflight_;
        }
        cv_.notify_all();
    }
}

}  // namespace mph

extern "C" int mph_format_e(const double* values, long long n, int as_float, char* out, long long capacity,
                            long long* length) {
    if (n < 0 || (n > 0 && (!values || !out)) || capacity < 0 || !length) return MPH_ERR_ARG;
    *length = 0;
    if (n == 0) return MPH_OK;
    double* dv = nullptr;
    char* dt = nullptr;
    int st = MPH_OK;
    std::vector<char> host((size_t)n * mph::kTextValueStride);
    if (cudaMalloc(&dv, (size_t)n * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dt, host.size()) != cudaSuccess ||
        cudaMemcpy(dv, values, (size_t)n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        st = MPH_ERR_CUDA;
    } else {
        mph::launch_text_values(dv, n, as_float, dt, 0);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpy(host.data(), dt, host.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
            st = MPH_ERR_CUDA;
    }
    cudaFree(dv);
    cudaFree(dt);
    if (st != MPH_OK) return st;
    long long k = 0;
    for (long long i = 0; i < n; ++i) {
        const char* rec = host.data() + i * mph::kTextValueStride;
        const int len = (unsigned char)rec[0];
        if (k + len > capacity) return MPH_ERR_CAPACITY;
        std::memcpy(out + k, rec + 1, (size_t)len);
        k += len;
    }
    *length = k;
    return MPH_OK;
}
