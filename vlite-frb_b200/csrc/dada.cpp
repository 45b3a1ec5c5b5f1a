// Shared-memory byte ring for the DADA-fed tools (host only).
//
// The reference's STATS and TS tools read their VDIF stream from a psrdada
// ring with ipcio_connect / ipcio_open('R') / ipcio_read / ipcbuf_eod
// (STATS:286-310, 444-462; TS:383-404, 767-826).  psrdada is not part of this
// build, so this is a project-defined ring with the same reader-side
// operations: one writer and one reader process share a POSIX shared-memory
// object named after the DADA key; the writer appends bytes and finally marks
// end of data; the reader gets the bytes in order, and a short read means end
// of data.  Every wait is bounded (timeout_ms) and reports VFRB_ERR_TIMEOUT.
// A reader can also take the bytes in place (acquire / release) from a
// mapping it page-locked (pin), so that vfrb_push_frames copies them to the
// device straight from the ring, with no host copy in between.
//
// As in a DADA ring, a header block (up to 4096 bytes of text the writer
// sets) sits beside the data block, and one reader at a time is the primary
// read client: vfrb_dada_open_read takes the role (ipcio_open 'R') and fails
// while another reader holds it; the ring's `iread` field names the holder
// (-1 = none), and vfrb_dada_force_iread clears it the way the reference
// tools do before opening (ipcbuf_force_iread, STATS:127-134, TS:140-147).
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include <atomic>
#include <new>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "vfrb.h"

namespace {

constexpr uint64_t kMagic = 0x7666726264616461ULL;  // "vfrbdada"

struct RingHdr {
  uint64_t magic;
  uint64_t cap;                    // data bytes (power of two)
  std::atomic<uint64_t> wpos;      // bytes written so far
  std::atomic<uint64_t> rpos;      // bytes consumed so far
  std::atomic<uint32_t> eod;       // writer finished
  std::atomic<int32_t> iread;      // primary read client's id, -1 = none
  std::atomic<uint32_t> hdr_len;   // header block length, kNoHeader until set
  uint32_t pad;
};
static_assert(sizeof(RingHdr) <= 64, "header fits one cache line");
constexpr size_t kHdrBytes = 64;
constexpr size_t kHeaderBlock = 4096;                 // the DADA header block
constexpr size_t kDataOff = kHdrBytes + kHeaderBlock;  // where the data block starts
constexpr uint32_t kNoHeader = 0xffffffffu;
std::atomic<int32_t> g_next_id{1};                    // reader ids of this process

void shm_name(uint32_t key, char* out, size_t n) { std::snprintf(out, n, "/vfrb_dada_%08x", key); }

void nap() {
  timespec ts{0, 100000};  // 0.1 ms
  nanosleep(&ts, nullptr);
}

double now_ms() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

}  // namespace

struct vfrb_dada {
  uint32_t key = 0;
  RingHdr* h = nullptr;
  uint8_t* data = nullptr;
  size_t map_bytes = 0;
  bool pinned = false;
  int32_t id = 0;        // this handle's reader id (pid-based, never -1)
  bool primary = false;  // holds the primary read client role
};

namespace {
int32_t new_reader_id() {
  return (int32_t)((((uint32_t)getpid() & 0x7fffu) << 16) | ((uint32_t)g_next_id.fetch_add(1) & 0xffffu));
}
}  // namespace

extern "C" {

int vfrb_dada_create(uint32_t key, uint64_t capacity, vfrb_dada** out) {
  if (!out || capacity < 4096 || (capacity & (capacity - 1))) return VFRB_ERR_ARG;
  char name[64];
  shm_name(key, name, sizeof name);
  const int fd = shm_open(name, O_CREAT | O_EXCL | O_RDWR, 0600);
  if (fd < 0) return VFRB_ERR;
  const size_t bytes = kDataOff + capacity;
  if (ftruncate(fd, (off_t)bytes) != 0) {
    close(fd);
    shm_unlink(name);
    return VFRB_ERR_NOMEM;
  }
  void* p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (p == MAP_FAILED) {
    shm_unlink(name);
    return VFRB_ERR_NOMEM;
  }
  auto* d = new vfrb_dada();
  d->key = key;
  d->h = new (p) RingHdr();
  d->h->cap = capacity;
  d->h->wpos.store(0);
  d->h->rpos.store(0);
  d->h->eod.store(0);
  d->h->iread.store(-1);
  d->h->hdr_len.store(kNoHeader);
  d->data = static_cast<uint8_t*>(p) + kDataOff;
  d->id = new_reader_id();
  d->map_bytes = bytes;
  std::atomic_thread_fence(std::memory_order_release);
  d->h->magic = kMagic;
  *out = d;
  return VFRB_OK;
}

int vfrb_dada_connect(uint32_t key, vfrb_dada** out) {
  if (!out) return VFRB_ERR_ARG;
  char name[64];
  shm_name(key, name, sizeof name);
  const int fd = shm_open(name, O_RDWR, 0600);
  if (fd < 0) return VFRB_ERR;
  struct stat sb;
  if (fstat(fd, &sb) != 0 || (size_t)sb.st_size < kDataOff + 4096) {
    close(fd);
    return VFRB_ERR;
  }
  void* p = mmap(nullptr, (size_t)sb.st_size, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
  close(fd);
  if (p == MAP_FAILED) return VFRB_ERR_NOMEM;
  auto* h = static_cast<RingHdr*>(p);
  if (h->magic != kMagic || kDataOff + h->cap != (size_t)sb.st_size) {
    munmap(p, (size_t)sb.st_size);
    return VFRB_ERR;
  }
  auto* d = new vfrb_dada();
  d->key = key;
  d->h = h;
  d->data = static_cast<uint8_t*>(p) + kDataOff;
  d->map_bytes = (size_t)sb.st_size;
  d->id = new_reader_id();
  *out = d;
  return VFRB_OK;
}

int64_t vfrb_dada_write(vfrb_dada* d, const void* bytes, uint64_t n, int timeout_ms) {
  if (!d || (!bytes && n)) return -VFRB_ERR_ARG;
  const uint64_t cap = d->h->cap;
  const auto* src = static_cast<const uint8_t*>(bytes);
  uint64_t done = 0;
  double t0 = now_ms();
  while (done < n) {
    const uint64_t w = d->h->wpos.load(std::memory_order_relaxed);
    const uint64_t r = d->h->rpos.load(std::memory_order_acquire);
    const uint64_t room = cap - (w - r);
    if (room == 0) {
      if (now_ms() - t0 > timeout_ms) return done ? (int64_t)done : -VFRB_ERR_TIMEOUT;
      nap();
      continue;
    }
    uint64_t k = n - done < room ? n - done : room;
    const uint64_t at = w & (cap - 1);
    if (k > cap - at) k = cap - at;
    std::memcpy(d->data + at, src + done, k);
    d->h->wpos.store(w + k, std::memory_order_release);
    done += k;
    t0 = now_ms();
  }
  return (int64_t)done;
}

int vfrb_dada_set_eod(vfrb_dada* d) {
  if (!d) return VFRB_ERR_ARG;
  d->h->eod.store(1, std::memory_order_release);
  return VFRB_OK;
}

int64_t vfrb_dada_read(vfrb_dada* d, void* buf, uint64_t n, int timeout_ms) {
  if (!d || (!buf && n)) return -VFRB_ERR_ARG;
  const uint64_t cap = d->h->cap;
  auto* dst = static_cast<uint8_t*>(buf);
  uint64_t done = 0;
  double t0 = now_ms();
  while (done < n) {
    const uint64_t r = d->h->rpos.load(std::memory_order_relaxed);
    const uint64_t w = d->h->wpos.load(std::memory_order_acquire);
    if (w == r) {
      if (d->h->eod.load(std::memory_order_acquire) && d->h->wpos.load(std::memory_order_acquire) == r) break;
      if (now_ms() - t0 > timeout_ms) return done ? (int64_t)done : -VFRB_ERR_TIMEOUT;
      nap();
      continue;
    }
    uint64_t k = w - r < n - done ? w - r : n - done;
    const uint64_t at = r & (cap - 1);
    if (k > cap - at) k = cap - at;
    std::memcpy(dst + done, d->data + at, k);
    d->h->rpos.store(r + k, std::memory_order_release);
    done += k;
    t0 = now_ms();
  }
  return (int64_t)done;
}

int64_t vfrb_dada_acquire(vfrb_dada* d, const uint8_t** ptr, uint64_t max_n, int timeout_ms) {
  if (!d || !ptr || max_n == 0) return -VFRB_ERR_ARG;
  const uint64_t cap = d->h->cap;
  const double t0 = now_ms();
  for (;;) {
    const uint64_t r = d->h->rpos.load(std::memory_order_relaxed);
    const uint64_t w = d->h->wpos.load(std::memory_order_acquire);
    if (w != r) {
      const uint64_t at = r & (cap - 1);
      uint64_t k = w - r;
      if (k > cap - at) k = cap - at;  // contiguous up to the ring's end
      if (k > max_n) k = max_n;
      *ptr = d->data + at;
      return (int64_t)k;
    }
    if (d->h->eod.load(std::memory_order_acquire) && d->h->wpos.load(std::memory_order_acquire) == r) {
      *ptr = nullptr;
      return 0;
    }
    if (now_ms() - t0 > timeout_ms) return -VFRB_ERR_TIMEOUT;
    nap();
  }
}

int vfrb_dada_release(vfrb_dada* d, uint64_t n) {
  if (!d) return VFRB_ERR_ARG;
  const uint64_t r = d->h->rpos.load(std::memory_order_relaxed);
  if (n > d->h->wpos.load(std::memory_order_acquire) - r) return VFRB_ERR_ARG;
  d->h->rpos.store(r + n, std::memory_order_release);
  return VFRB_OK;
}

int vfrb_dada_pin(vfrb_dada* d) {
  if (!d) return VFRB_ERR_ARG;
  if (d->pinned) return VFRB_OK;
  if (cudaHostRegister(d->h, d->map_bytes, cudaHostRegisterDefault) != cudaSuccess) {
    cudaGetLastError();
    return VFRB_ERR_CUDA;
  }
  d->pinned = true;
  return VFRB_OK;
}

int vfrb_dada_eod(const vfrb_dada* d) {
  if (!d) return VFRB_ERR_ARG;
  return d->h->eod.load(std::memory_order_acquire) &&
         d->h->wpos.load(std::memory_order_acquire) == d->h->rpos.load(std::memory_order_acquire);
}

int vfrb_dada_set_header(vfrb_dada* d, const char* text, uint64_t n) {
  if (!d || (!text && n) || n > kHeaderBlock) return VFRB_ERR_ARG;
  std::memcpy(reinterpret_cast<uint8_t*>(d->h) + kHdrBytes, text, n);
  d->h->hdr_len.store((uint32_t)n, std::memory_order_release);
  return VFRB_OK;
}

int64_t vfrb_dada_get_header(vfrb_dada* d, char* buf, uint64_t cap, int timeout_ms) {
  if (!d || (!buf && cap)) return -VFRB_ERR_ARG;
  const double t0 = now_ms();
  uint32_t n;
  while ((n = d->h->hdr_len.load(std::memory_order_acquire)) == kNoHeader) {
    if (now_ms() - t0 > timeout_ms) return -VFRB_ERR_TIMEOUT;
    nap();
  }
  std::memcpy(buf, reinterpret_cast<const uint8_t*>(d->h) + kHdrBytes, n < cap ? n : cap);
  return (int64_t)n;
}

int vfrb_dada_iread(const vfrb_dada* d) { return d ? (int)d->h->iread.load(std::memory_order_acquire) : -1; }

int vfrb_dada_force_iread(vfrb_dada* d) {
  if (!d) return -1;
  return (int)d->h->iread.exchange(-1, std::memory_order_acq_rel);
}

int vfrb_dada_open_read(vfrb_dada* d) {
  if (!d) return VFRB_ERR_ARG;
  if (d->primary) return VFRB_OK;
  int32_t none = -1;
  if (!d->h->iread.compare_exchange_strong(none, d->id, std::memory_order_acq_rel)) return VFRB_ERR;
  d->primary = true;
  return VFRB_OK;
}

int vfrb_dada_close(vfrb_dada* d) {
  if (!d) return VFRB_ERR_ARG;
  if (d->primary) {  // give the role back unless it was forced away meanwhile
    int32_t me = d->id;
    d->h->iread.compare_exchange_strong(me, -1, std::memory_order_acq_rel);
  }
  if (d->pinned && cudaHostUnregister(d->h) != cudaSuccess) cudaGetLastError();
  munmap(d->h, d->map_bytes);
  delete d;
  return VFRB_OK;
}

int vfrb_dada_destroy(uint32_t key) {
  char name[64];
  shm_name(key, name, sizeof name);
  return shm_unlink(name) == 0 ? VFRB_OK : VFRB_ERR;
}

}  // extern "C"
