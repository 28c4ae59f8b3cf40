// mph_text.h — device-side *.prof / *.vtk text (k_text.cu) and the host
// writer thread that copies it out and writes the file (mph_text.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

namespace mph {

// Record kinds: one particle's text in a section.
enum TextRecord : int {
    kRecNone = 0,     // header-only section
    kRecProf = 1,     // "%d %e %e %e  %e %e %e\n": src2 type, src0 pos (double4), src1 vel (double4)
    kRecVec3f = 2,    // "%e %e %e\n" of (float) x, y, z of src0 (double4)
    kRecScalarf = 3,  // "%e\n" of (float) src0[i] (double)
    kRecScalard = 4,  // "%e\n" of src0[i] (double)
    kRecInt = 5,      // "%d\n" of src0[i] (int)
    kRecCell = 6,     // "1 %d " of the record index
    kRecOne = 7,      // "1 "
    kRecKinds = 8
};

// Longest text of one record of each kind ("%e" of a double is at most 14
// characters, of a float 13; "%d" at most 11).
constexpr int kTextMaxRecord[kRecKinds] = {0, 103, 42, 14, 15, 12, 14, 2};
constexpr int kTextMaxUnit = 256;     // a header or a record
constexpr int kTextBlockUnits = 256;  // units (a header or a record) per block of the text kernels
constexpr int kTextMaxSections = 12;
constexpr int kTextHeadPool = 1536;
constexpr int kTextValueStride = 16;  // mph_format_e: a length byte + at most 15 characters

struct TextSection {
    int kind;
    int n;            // records
    int head_off;     // header bytes in TextDoc::head
    int head_len;
    int first_block;  // set by text_blocks
    const void* src0;
    const void* src1;
    const void* src2;
};

struct TextDoc {
    int nsec;
    int nblocks;
    int head_used;
    TextSection sec[kTextMaxSections];
    char head[kTextHeadPool];
};

// Appends a section; false if the header pool or the section table is full.
bool text_add(TextDoc& d, const char* head, int kind, int n, const void* src0 = nullptr,
              const void* src1 = nullptr, const void* src2 = nullptr);
int text_blocks(TextDoc& d);                 // assigns blocks; returns the grid size
size_t text_max_bytes(const TextDoc& d);     // an upper bound of the document's bytes
// Three launches on s: per-block byte counts, their scan (off[nblocks] = total
// bytes), the formatted text into out.  Returns the number of launches.
// off has nblocks + 2 entries: off[nblocks + 1] != 0 flags a record whose text
// did not have the length counted for it.
int launch_text(const TextDoc& d, uint16_t* unit_len, uint32_t* blk_bytes, unsigned long long* off, char* out,
                cudaStream_t s);
void launch_text_values(const double* v, long long n, int as_float, char* out, cudaStream_t s);

// Formats documents on the caller's stream and writes them to files from a
// worker thread, with two device text buffers so that the next document can
// be formatted while the previous one is copied out and written.
class TextWriter {
  public:
    explicit TextWriter(int device);
    ~TextWriter();  // writes every submitted document, then stops
    TextWriter(const TextWriter&) = delete;
    TextWriter& operator=(const TextWriter&) = delete;

    // Enqueues doc's formatting on `stream` (after the work already there)
    // and its write to `path`.  Returns MPH_OK or a status with *err set.
    int submit(TextDoc& doc, cudaStream_t stream, const std::string& path, std::string* err, int* launches);
    // Waits for every submitted write; returns the first failure since the
    // last wait (MPH_OK if none) with its message in *err.
    int wait(std::string* err);

  private:
    struct Slot {
        char* text = nullptr;
        size_t cap = 0;
        uint32_t* blk = nullptr;
        uint16_t* unit_len = nullptr;
        unsigned long long* off = nullptr;
        int blk_cap = 0;
        cudaEvent_t done = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        int nblocks;
        std::string path;
    };
    void run();
    void fail(int code, const std::string& msg);

    int device_;
    Slot slot_[2];
    int next_ = 0;
    cudaStream_t copy_ = nullptr;
    char* pinned_ = nullptr;
    size_t pinned_cap_ = 0;
    unsigned long long* total_ = nullptr;  // pinned: {bytes, length-mismatch flag}
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Job> q_;
    int inflight_ = 0;
    bool stop_ = false;
    int err_code_ = 0;
    std::string err_msg_;
    std::thread th_;
};

}  // namespace mph
