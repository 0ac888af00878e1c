// psb_store.cu -- the segment store of the out-of-core search (host code).
//
// Restates the reference's Store (Common/Store.h:13-178, Common/Store.cpp):
// numbered segments, each a list of chunks that are read back in the order
// they were written.  A file store spreads the segments round-robin over
// several directories (ParallelStoreImpl, Store.cpp:254-296); in each
// directory either
//   files_per_path == 0: one file per segment, <dir>/<name>_<segment>
//                        (MultiFileStoreImpl, :190-252);
//   files_per_path == 1: one file, <dir>/<name> (SingleFileStoreImpl, :89-188);
//   files_per_path == k: k files <dir>/<name>_p<i>, file i holding the
//                        segments s with s * k / max_segments == i
//                        (SequentialStoreImpl, :298-344).
// A file is created at its first write and removed as soon as none of its
// segments holds data (or when the store is destroyed), so a file of
// consecutive segments disappears once the search has moved past them.  The
// chunk lists live in host memory; the files hold the raw chunk bytes,
// appended.  A memory store (no directories) keeps the chunks in host memory
// instead.  File errors are returned (PSB_ERR_IO), not fatal.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cerrno>
#include <cstring>
#include <filesystem>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/psb200.h"
#include "psb_internal.h"

namespace psb {

namespace {

int io_error(const std::string& what, const std::string& path) {
    return psb_set_error(PSB_ERR_IO, (what + " " + path + ": " + std::strerror(errno)).c_str());
}

struct Chunk {
    uint64_t offset;  // in the file (file stores) or index into the memory chunks
    uint64_t length;
    int64_t next;
};

// Chunk lists of a set of segments: head / tail / read pointer per segment.
struct ChunkLists {
    std::vector<Chunk> chunks;
    std::vector<int64_t> head, tail, rd;
    int nonempty = 0;
    explicit ChunkLists(int n) : head(n, -1), tail(n, -1), rd(n, -1) {}
    void append(int s, uint64_t offset, uint64_t length) {
        const int64_t pos = int64_t(chunks.size());
        chunks.push_back(Chunk{offset, length, -1});
        if (head[s] < 0) {
            head[s] = tail[s] = rd[s] = pos;
            nonempty++;
        } else {
            chunks[size_t(tail[s])].next = pos;
            tail[s] = pos;
        }
    }
    uint64_t length(int s) const {
        uint64_t n = 0;
        for (int64_t p = head[s]; p >= 0; p = chunks[size_t(p)].next) n += chunks[size_t(p)].length;
        return n;
    }
    bool drop(int s) {  // true if s held data
        if (head[s] < 0) return false;
        head[s] = tail[s] = rd[s] = -1;
        nonempty--;
        return true;
    }
    void clear() {
        chunks.clear();
        std::fill(head.begin(), head.end(), -1);
        std::fill(tail.begin(), tail.end(), -1);
        std::fill(rd.begin(), rd.end(), -1);
        nonempty = 0;
    }
};

}  // namespace

class StoreImpl {
public:
    virtual ~StoreImpl() = default;
    virtual uint64_t length(int s) const = 0;
    virtual uint64_t total() const = 0;
    virtual void rewind(int s) = 0;
    virtual int write(int s, const void* buf, uint64_t size) = 0;
    // Next chunk of s into buf (cap bytes); *got = 0 past the last chunk.
    virtual int read(int s, void* buf, uint64_t cap, uint64_t* got) = 0;
    virtual int erase(int s) = 0;
    virtual int erase_all() = 0;
};

// One file holding chunks of segments [0, n) (SingleFileStoreImpl).
class FileStore : public StoreImpl {
public:
    FileStore(int n, std::string path) : path_(std::move(path)), lists_(n) {}
    ~FileStore() override { erase_all(); }
    uint64_t length(int s) const override { return lists_.length(s); }
    uint64_t total() const override { return size_; }
    void rewind(int s) override { lists_.rd[s] = lists_.head[s]; }
    int write(int s, const void* buf, uint64_t size) override {
        std::lock_guard<std::mutex> g(mu_);
        if (fd_ < 0) {  // first chunk since the file was last empty: create it afresh
            fd_ = ::open(path_.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0644);
            if (fd_ < 0) return io_error("cannot create", path_);
            size_ = 0;
        }
        const char* p = static_cast<const char*>(buf);
        for (uint64_t done = 0; done < size;) {
            const ssize_t w = ::pwrite(fd_, p + done, size - done, off_t(size_ + done));
            if (w <= 0) return io_error("cannot write", path_);
            done += uint64_t(w);
        }
        lists_.append(s, size_, size);
        size_ += size;
        return PSB_OK;
    }
    int read(int s, void* buf, uint64_t cap, uint64_t* got) override {
        *got = 0;
        const int64_t pos = lists_.rd[s];
        if (pos < 0) return PSB_OK;
        const Chunk& c = lists_.chunks[size_t(pos)];
        if (c.length > cap) return psb_set_error(PSB_ERR_CAPACITY, "store chunk larger than the read buffer");
        char* p = static_cast<char*>(buf);
        for (uint64_t done = 0; done < c.length;) {
            const ssize_t r = ::pread(fd_, p + done, c.length - done, off_t(c.offset + done));
            if (r <= 0) return io_error("cannot read", path_);
            done += uint64_t(r);
        }
        lists_.rd[s] = c.next;
        *got = c.length;
        return PSB_OK;
    }
    int erase(int s) override {
        std::lock_guard<std::mutex> g(mu_);
        lists_.drop(s);
        return lists_.nonempty == 0 ? remove_file() : PSB_OK;
    }
    int erase_all() override {
        std::lock_guard<std::mutex> g(mu_);
        lists_.clear();
        return remove_file();
    }

private:
    int remove_file() {
        lists_.clear();
        size_ = 0;
        if (fd_ < 0) return PSB_OK;
        ::close(fd_);
        fd_ = -1;
        if (::unlink(path_.c_str()) != 0 && errno != ENOENT) return io_error("cannot delete", path_);
        return PSB_OK;
    }
    std::string path_;
    ChunkLists lists_;
    int fd_ = -1;
    uint64_t size_ = 0;
    std::mutex mu_;
};

// Chunks in host memory.
class MemoryStore : public StoreImpl {
public:
    explicit MemoryStore(int n) : lists_(n), data_(n) {}
    uint64_t length(int s) const override { return lists_.length(s); }
    uint64_t total() const override { return total_; }
    void rewind(int s) override { lists_.rd[s] = lists_.head[s]; }
    int write(int s, const void* buf, uint64_t size) override {
        std::lock_guard<std::mutex> g(mu_);
        const char* p = static_cast<const char*>(buf);
        try {
            data_[size_t(s)].emplace_back(p, p + size);
        } catch (const std::bad_alloc&) {
            return psb_set_error(PSB_ERR_NOMEM, "segment store: host memory");
        }
        lists_.append(s, data_[size_t(s)].size() - 1, size);
        total_ += size;
        return PSB_OK;
    }
    int read(int s, void* buf, uint64_t cap, uint64_t* got) override {
        *got = 0;
        const int64_t pos = lists_.rd[s];
        if (pos < 0) return PSB_OK;
        const Chunk& c = lists_.chunks[size_t(pos)];
        if (c.length > cap) return psb_set_error(PSB_ERR_CAPACITY, "store chunk larger than the read buffer");
        std::memcpy(buf, data_[size_t(s)][c.offset].data(), c.length);
        lists_.rd[s] = c.next;
        *got = c.length;
        return PSB_OK;
    }
    int erase(int s) override {
        std::lock_guard<std::mutex> g(mu_);
        total_ -= lists_.length(s);
        lists_.drop(s);
        std::vector<std::vector<char>>().swap(data_[size_t(s)]);
        if (lists_.nonempty == 0) lists_.clear();
        return PSB_OK;
    }
    int erase_all() override {
        std::lock_guard<std::mutex> g(mu_);
        lists_.clear();
        for (auto& d : data_) std::vector<std::vector<char>>().swap(d);
        total_ = 0;
        return PSB_OK;
    }

private:
    ChunkLists lists_;
    std::vector<std::vector<std::vector<char>>> data_;
    uint64_t total_ = 0;
    std::mutex mu_;
};

// Segments routed to member stores: round-robin over directories
// (parallel) or in consecutive ranges over the files of one directory
// (sequential), or one file per segment.
class RoutedStore : public StoreImpl {
public:
    enum Route { kRoundRobin, kRanges, kOwn };
    RoutedStore(int n, Route r, std::vector<std::unique_ptr<StoreImpl>> parts)
        : n_(n), route_(r), parts_(std::move(parts)) {}
    uint64_t length(int s) const override { return part(s).length(local(s)); }
    uint64_t total() const override {
        uint64_t t = 0;
        for (const auto& p : parts_) t += p->total();
        return t;
    }
    void rewind(int s) override { part(s).rewind(local(s)); }
    int write(int s, const void* buf, uint64_t size) override { return part(s).write(local(s), buf, size); }
    int read(int s, void* buf, uint64_t cap, uint64_t* got) override { return part(s).read(local(s), buf, cap, got); }
    int erase(int s) override { return part(s).erase(local(s)); }
    int erase_all() override {
        int rc = PSB_OK;
        for (auto& p : parts_)
            if (int r = p->erase_all()) rc = r;
        return rc;
    }

private:
    size_t index(int s) const {
        const size_t k = parts_.size();
        return route_ == kRoundRobin ? size_t(s) % k : route_ == kRanges ? size_t(s) * k / size_t(n_) : size_t(s);
    }
    int local(int s) const { return route_ == kOwn ? 0 : s; }
    StoreImpl& part(int s) { return *parts_[index(s)]; }
    const StoreImpl& part(int s) const { return *parts_[index(s)]; }
    int n_;
    Route route_;
    std::vector<std::unique_ptr<StoreImpl>> parts_;
};

// Store::CreateFileStore (Store.cpp:400-417), or a memory store without directories.
int store_create(int n, const std::string& name, const std::vector<std::string>& dirs, int files_per_path,
                 StorePtr* out) {
    if (n <= 0) return psb_set_error(PSB_ERR_ARG, "store: max_segments must be positive");
    if (files_per_path < 0) return psb_set_error(PSB_ERR_ARG, "store: files_per_path must be >= 0");
    if (dirs.empty()) {
        out->reset(new MemoryStore(n));
        return PSB_OK;
    }
    std::vector<std::unique_ptr<StoreImpl>> per_dir;
    for (const std::string& d : dirs) {
        std::error_code ec;
        std::filesystem::create_directories(d, ec);
        if (ec) return psb_set_error(PSB_ERR_IO, ("cannot create directory " + d + ": " + ec.message()).c_str());
        const std::string base = d + "/" + name;
        if (files_per_path == 1) {
            per_dir.push_back(std::make_unique<FileStore>(n, base));
        } else if (files_per_path == 0) {
            std::vector<std::unique_ptr<StoreImpl>> files;
            for (int s = 0; s < n; s++) files.push_back(std::make_unique<FileStore>(1, base + "_" + std::to_string(s)));
            per_dir.push_back(std::make_unique<RoutedStore>(n, RoutedStore::kOwn, std::move(files)));
        } else {
            std::vector<std::unique_ptr<StoreImpl>> files;
            for (int i = 0; i < files_per_path; i++)
                files.push_back(std::make_unique<FileStore>(n, base + "_p" + std::to_string(i)));
            per_dir.push_back(std::make_unique<RoutedStore>(n, RoutedStore::kRanges, std::move(files)));
        }
    }
    out->reset(new RoutedStore(n, RoutedStore::kRoundRobin, std::move(per_dir)));
    return PSB_OK;
}

uint64_t store_length(const StoreImpl& s, int segment) { return s.length(segment); }
uint64_t store_total(const StoreImpl& s) { return s.total(); }
void store_rewind(StoreImpl& s, int segment) { s.rewind(segment); }
int store_write(StoreImpl& s, int segment, const void* buf, uint64_t size) {
    return size ? s.write(segment, buf, size) : PSB_OK;  // Store::Write skips empty chunks (Store.cpp:44-52)
}
int store_read(StoreImpl& s, int segment, void* buf, uint64_t cap, uint64_t* got) {
    return s.read(segment, buf, cap, got);
}
int store_erase(StoreImpl& s, int segment) { return s.erase(segment); }
int store_erase_all(StoreImpl& s) { return s.erase_all(); }
void store_destroy(StoreImpl* s) { delete s; }

}  // namespace psb

struct psb_store {
    psb::StorePtr impl;
    int n = 0;
};

namespace {
bool bad_segment(const psb_store* st, int s) { return !st || s < 0 || s >= st->n; }
}  // namespace

extern "C" {

int psb_store_create(int max_segments, const char* name, const char* const* directories, int n_directories,
                     int files_per_path, psb_store** out) {
    if (!out || !name || !*name || n_directories < 0 || (n_directories && !directories))
        return psb_set_error(PSB_ERR_ARG, "bad argument");
    std::vector<std::string> dirs;
    for (int i = 0; i < n_directories; i++) {
        if (!directories[i] || !*directories[i]) return psb_set_error(PSB_ERR_ARG, "empty directory name");
        dirs.emplace_back(directories[i]);
    }
    auto st = std::make_unique<psb_store>();
    st->n = max_segments;
    if (int rc = psb::store_create(max_segments, name, dirs, files_per_path, &st->impl)) return rc;
    *out = st.release();
    return PSB_OK;
}

int psb_store_destroy(psb_store* st) {
    if (!st) return PSB_OK;
    const int rc = st->impl->erase_all();
    delete st;
    return rc;
}

int psb_store_write(psb_store* st, int segment, const void* buf, uint64_t size) {
    if (bad_segment(st, segment) || (size && !buf)) return psb_set_error(PSB_ERR_ARG, "bad argument");
    return psb::store_write(*st->impl, segment, buf, size);
}

int psb_store_read(psb_store* st, int segment, void* buf, uint64_t cap, uint64_t* got) {
    if (bad_segment(st, segment) || !got || (cap && !buf)) return psb_set_error(PSB_ERR_ARG, "bad argument");
    return st->impl->read(segment, buf, cap, got);
}

int psb_store_rewind(psb_store* st, int segment) {
    if (bad_segment(st, segment)) return psb_set_error(PSB_ERR_ARG, "bad argument");
    st->impl->rewind(segment);
    return PSB_OK;
}

int psb_store_length(const psb_store* st, int segment, uint64_t* bytes) {
    if (!st || !bytes || segment >= st->n) return psb_set_error(PSB_ERR_ARG, "bad argument");
    *bytes = segment < 0 ? st->impl->total() : st->impl->length(segment);
    return PSB_OK;
}

int psb_store_delete(psb_store* st, int segment) {
    if (!st || segment >= st->n) return psb_set_error(PSB_ERR_ARG, "bad argument");
    return segment < 0 ? st->impl->erase_all() : st->impl->erase(segment);
}

}  // extern "C"
