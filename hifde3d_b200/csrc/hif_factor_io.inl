// Factor save / load: the factorization held by an Engine written to a file and
// read back into another handle of the same N, P and partition, so that a
// serving process can start with operators factored elsewhere (or earlier)
// instead of refactoring them. The reference keeps its factor only in memory
// (FactorData / IndexData per block, include/data.hpp:11-62,84-110, held in
// HIFFactor::schur_level_data_ / skel_level_data_, include/Factor.hpp:201-202);
// this file format is this library's own.
//
// Layout (host byte order, checked on load by a marker word):
//   header   "HIFB200F", u32 version, u32 0x01020304, i32 N, P, partition, L,
//            symmetric, precision the factor was made in (informational),
//            has_operator, nsteps, f64 eps, i64 NC^3
//   per step (Schur or skeletonization phase of one level)
//            i32 level, kind (bit 0: skeletonization; bit 1: eliminated by
//            Cholesky, so the arena holds L | L^-1 | Y | W), cells_per_dir,
//            nblocks; i64 arena doubles, n_red,
//            n_skel; per block i32 face, cell, nbr and the int vectors
//            global, red_pos, skel_pos, jpvt and the double vector rdiag
//            (each an i64 count then the values); the i64 offset vectors
//            o_a22, o_inv, o_x, o_w, o_red, o_skel; the red and skel DOF lists
//            (n_red, n_skel ints); the arena (A22 | A22^-1 | X | W per block)
//   operator 7 NC^3 doubles (the stencil bands) when has_operator
//   trailer  u64 checksum of every byte before it
// Everything read is validated before any device access uses it: sizes,
// offsets inside the phase's arena, DOF ids inside [0, NC^3), and the checksum
// over the whole file; a file that fails any check leaves the handle without a
// factorization and returns HIF_ERR_IO.

constexpr char kFactorMagic[8] = {'H', 'I', 'F', 'B', '2', '0', '0', 'F'};
constexpr uint32_t kFactorVersion = 1;
constexpr uint32_t kFactorEndian = 0x01020304u;
constexpr size_t kIoChunk = size_t(64) << 20;  // bytes per host <-> device transfer

// Word-wise checksum (64-bit multiply-rotate over 8-byte words, then the tail
// bytes); order-dependent, so a swapped or truncated section changes it.
struct IoHash {
  uint64_t h = 0x9E3779B97F4A7C15ull;
  unsigned char tail[8];
  int nt = 0;
  void word(uint64_t w) {
    h ^= w;
    h *= 0xFF51AFD7ED558CCDull;
    h = (h << 29) | (h >> 35);
  }
  void add(const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    while (n > 0 && nt > 0 && nt < 8) {
      tail[nt++] = *c++;
      --n;
      if (nt == 8) {
        uint64_t w;
        std::memcpy(&w, tail, 8);
        word(w);
        nt = 0;
      }
    }
    while (n >= 8) {
      uint64_t w;
      std::memcpy(&w, c, 8);
      word(w);
      c += 8;
      n -= 8;
    }
    while (n > 0) {
      tail[nt++] = *c++;
      --n;
    }
  }
  uint64_t value() const {
    IoHash t = *this;
    uint64_t w = 0;
    std::memcpy(&w, t.tail, t.nt);
    t.word(w ^ ((uint64_t)t.nt << 56));
    return t.h;
  }
};

[[noreturn]] void io_fail(const std::string& what) { throw Error{HIF_ERR_IO, what}; }

// Writes `path` + ".tmp" and renames it to `path` once complete, so a failed
// save never leaves a partial factor under the target name.
class FactorWriter {
 public:
  explicit FactorWriter(const char* path)
      : path_(path), tmp_(std::string(path) + ".tmp") {
    f_ = std::fopen(tmp_.c_str(), "wb");
    if (!f_) io_fail("cannot open " + tmp_ + " for writing");
  }
  ~FactorWriter() {
    if (f_) {  // not finished: drop the partial file
      std::fclose(f_);
      std::remove(tmp_.c_str());
    }
    if (pin_) cudaFreeHost(pin_);
  }
  void raw(const void* p, size_t n) {
    if (n == 0) return;
    hash_.add(p, n);
    if (std::fwrite(p, 1, n, f_) != n) io_fail("write failed: " + tmp_);
  }
  template <class T>
  void pod(const T& v) {
    raw(&v, sizeof(T));
  }
  template <class T>
  void vec(const std::vector<T>& v) {
    pod<long long>((long long)v.size());
    raw(v.data(), v.size() * sizeof(T));
  }
  // device array of `count` T, streamed through pinned host memory
  template <class T>
  void device(const T* d, long long count, cudaStream_t s) {
    const size_t total = (size_t)count * sizeof(T);
    if (total == 0) return;
    if (!pin_) HIF_CK(cudaMallocHost(&pin_, kIoChunk));
    for (size_t off = 0; off < total; off += kIoChunk) {
      const size_t n = std::min(kIoChunk, total - off);
      HIF_CK(cudaMemcpyAsync(pin_, reinterpret_cast<const char*>(d) + off, n,
                             cudaMemcpyDeviceToHost, s));
      HIF_CK(cudaStreamSynchronize(s));
      raw(pin_, n);
    }
  }
  void finish() {
    const uint64_t c = hash_.value();
    if (std::fwrite(&c, 1, 8, f_) != 8 || std::fflush(f_) != 0)
      io_fail(std::string("write failed: ") + path_);
    const int rc = std::fclose(f_);
    f_ = nullptr;
    if (rc != 0 || std::rename(tmp_.c_str(), path_.c_str()) != 0) {
      std::remove(tmp_.c_str());
      io_fail(std::string("cannot complete ") + path_);
    }
  }

 private:
  std::FILE* f_ = nullptr;
  std::string path_, tmp_;
  IoHash hash_;
  void* pin_ = nullptr;
};

class FactorReader {
 public:
  explicit FactorReader(const char* path) : f_(std::fopen(path, "rb")), path_(path) {
    if (!f_) io_fail(std::string("cannot open ") + path);
  }
  ~FactorReader() {
    if (f_) std::fclose(f_);
    if (pin_) cudaFreeHost(pin_);
  }
  void raw(void* p, size_t n) {
    if (n == 0) return;
    if (std::fread(p, 1, n, f_) != n) io_fail(std::string("truncated factor file: ") + path_);
    hash_.add(p, n);
  }
  template <class T>
  T pod() {
    T v;
    raw(&v, sizeof(T));
    return v;
  }
  // a vector of at most `max_count` entries
  template <class T>
  std::vector<T> vec(long long max_count) {
    const long long n = pod<long long>();
    if (n < 0 || n > max_count) io_fail("corrupt factor file: vector length out of range");
    std::vector<T> v((size_t)n);
    raw(v.data(), (size_t)n * sizeof(T));
    return v;
  }
  template <class T>
  void device(T* d, long long count, cudaStream_t s) {
    const size_t total = (size_t)count * sizeof(T);
    if (total == 0) return;
    if (!pin_) HIF_CK(cudaMallocHost(&pin_, kIoChunk));
    for (size_t off = 0; off < total; off += kIoChunk) {
      const size_t n = std::min(kIoChunk, total - off);
      HIF_CK(cudaStreamSynchronize(s));  // the previous chunk has left pin_
      raw(pin_, n);
      HIF_CK(cudaMemcpyAsync(reinterpret_cast<char*>(d) + off, pin_, n, cudaMemcpyHostToDevice, s));
    }
    HIF_CK(cudaStreamSynchronize(s));
  }
  void finish() {
    const uint64_t want = hash_.value();
    uint64_t got = 0;
    if (std::fread(&got, 1, 8, f_) != 8) io_fail(std::string("truncated factor file: ") + path_);
    if (got != want) io_fail(std::string("factor file checksum mismatch: ") + path_);
    char extra;
    if (std::fread(&extra, 1, 1, f_) != 0)
      io_fail(std::string("trailing bytes after the factor: ") + path_);
  }

 private:
  std::FILE* f_;
  std::string path_;
  IoHash hash_;
  void* pin_ = nullptr;
};

// Doubles of a phase's arena: the end of the furthest matrix of any block.
inline long long step_arena_doubles(const StepData& st) {
  long long asz = 0;
  for (size_t b = 0; b < st.blocks.size(); ++b) {
    const long long r = st.blocks[b].r(), s = st.blocks[b].s();
    asz = std::max(asz, st.o_a22[b] + r * r);
    asz = std::max(asz, st.o_inv[b] + r * r);
    asz = std::max(asz, st.o_x[b] + r * s);
    if (st.skel) asz = std::max(asz, st.o_w[b] + s * r);
  }
  return asz;
}

void save_factor(Engine& e, const char* path) {
  if (!e.factored) throw Error{HIF_ERR_STATE, "save before Factor"};
  e.sync();
  FactorWriter w(path);
  w.raw(kFactorMagic, 8);
  w.pod<uint32_t>(kFactorVersion);
  w.pod<uint32_t>(kFactorEndian);
  const int32_t hdr[8] = {e.N, e.P, e.partition, e.L, e.symmetric ? 1 : 0, e.factor_precision,
                          e.have_op ? 1 : 0, (int32_t)e.steps.size()};
  w.raw(hdr, sizeof(hdr));
  w.pod<double>(e.eps);
  w.pod<long long>(e.n3);
  for (const StepData& st : e.steps) {
    const int32_t sh[4] = {st.level, (st.skel ? 1 : 0) | (st.chol ? 2 : 0), st.cpd,
                           (int32_t)st.blocks.size()};
    w.raw(sh, sizeof(sh));
    const long long asz = step_arena_doubles(st);
    w.pod<long long>(asz);
    w.pod<long long>(st.n_red);
    w.pod<long long>(st.n_skel);
    for (const BlockInfo& b : st.blocks) {
      const int32_t bh[3] = {b.face, b.cell, b.nbr};
      w.raw(bh, sizeof(bh));
      w.vec(b.global);
      w.vec(b.red_pos);
      w.vec(b.skel_pos);
      w.vec(b.jpvt);
      w.vec(b.rdiag);
    }
    w.vec(st.o_a22);
    w.vec(st.o_inv);
    w.vec(st.o_x);
    w.vec(st.o_w);
    w.vec(st.o_red);
    w.vec(st.o_skel);
    w.device(st.d_red, st.n_red, e.stream);
    w.device(st.d_skel, st.n_skel, e.stream);
    w.device(st.arena, asz, e.stream);
  }
  if (e.have_op) w.device(e.d_band, 7 * e.n3, e.stream);
  w.finish();
}

void load_factor(Engine& e, const char* path) {
  e.sync();
  e.join_face_partition();
  e.join_cell_partition();
  e.initialize();  // drops any factorization the handle held
  FactorReader rd(path);
  bool op_touched = false;
  try {
    char magic[8];
    rd.raw(magic, 8);
    if (std::memcmp(magic, kFactorMagic, 8) != 0) io_fail(std::string("not a factor file: ") + path);
    if (rd.pod<uint32_t>() != kFactorVersion) io_fail("unsupported factor file version");
    if (rd.pod<uint32_t>() != kFactorEndian) io_fail("factor file written with another byte order");
    int32_t hdr[8];
    rd.raw(hdr, sizeof(hdr));
    if (hdr[0] != e.N || hdr[1] != e.P || hdr[2] != e.partition)
      throw Error{HIF_ERR_ARG, "factor file is for N=" + std::to_string(hdr[0]) + " P=" +
                                   std::to_string(hdr[1]) + " partition=" + std::to_string(hdr[2]) +
                                   ", the handle for N=" + std::to_string(e.N) + " P=" +
                                   std::to_string(e.P) + " partition=" +
                                   std::to_string(e.partition)};
    if (hdr[3] != e.L) io_fail("corrupt factor file: level count");
    const bool symmetric = hdr[4] != 0;
    const int factor_precision = hdr[5];
    const bool has_op = hdr[6] != 0;
    const int nsteps = hdr[7];
    if (nsteps < 0 || nsteps > 2 * e.L) io_fail("corrupt factor file: phase count");
    const double eps = rd.pod<double>();
    if (eps != e.eps)
      throw Error{HIF_ERR_ARG, "factor file was made with epsilon " + std::to_string(eps) +
                                   ", the handle's is " + std::to_string(e.eps)};
    if (rd.pod<long long>() != e.n3) io_fail("corrupt factor file: grid size");
    const long long n3 = e.n3;
    for (int q = 0; q < nsteps; ++q) {
      StepData st;
      int32_t sh[4];
      rd.raw(sh, sizeof(sh));
      st.level = sh[0];
      st.skel = (sh[1] & 1) != 0;
      st.chol = (sh[1] & 2) != 0;
      st.cpd = sh[2];
      const int nb = sh[3];
      if (st.level < 0 || st.level >= e.L || sh[1] < 0 || sh[1] > 3 || nb < 0 || nb > n3 ||
          (st.chol && !symmetric))
        io_fail("corrupt factor file: phase header");
      for (const StepData& o : e.steps)
        if (o.level == st.level && o.skel == st.skel) io_fail("corrupt factor file: repeated phase");
      const long long asz = rd.pod<long long>();
      st.n_red = rd.pod<long long>();
      st.n_skel = rd.pod<long long>();
      st.blocks.resize(nb);
      for (BlockInfo& b : st.blocks) {
        int32_t bh[3];
        rd.raw(bh, sizeof(bh));
        b.face = bh[0];
        b.cell = bh[1];
        b.nbr = bh[2];
        b.global = rd.vec<int>(n3);
        const long long ng = b.global.size();
        b.red_pos = rd.vec<int>(ng);
        b.skel_pos = rd.vec<int>(ng);
        b.jpvt = rd.vec<int>(ng);
        b.rdiag = rd.vec<double>(ng);
        for (int g : b.global)
          if (g < 0 || g >= n3) io_fail("corrupt factor file: DOF id out of range");
        for (const std::vector<int>* v : {&b.red_pos, &b.skel_pos, &b.jpvt})
          for (int p : *v)
            if (p < 0 || p >= ng) io_fail("corrupt factor file: block position out of range");
      }
      st.o_a22 = rd.vec<long long>(nb);
      st.o_inv = rd.vec<long long>(nb);
      st.o_x = rd.vec<long long>(nb);
      st.o_w = rd.vec<long long>(nb);
      st.o_red = rd.vec<long long>(nb);
      st.o_skel = rd.vec<long long>(nb);
      for (const std::vector<long long>* v : {&st.o_a22, &st.o_inv, &st.o_x, &st.o_w, &st.o_red,
                                              &st.o_skel})
        if ((long long)v->size() != nb) io_fail("corrupt factor file: offset table length");
      // the arena and the DOF lists are packed block after block: their sizes
      // follow from the block sizes, which bounds every allocation below
      long long packed = 0, sum_r = 0, sum_s = 0;
      for (int b = 0; b < nb; ++b) {
        const long long r = st.blocks[b].r(), s = st.blocks[b].s();
        packed += 2 * r * r + r * s + (st.skel ? s * r : 0);
        sum_r += r;
        sum_s += s;
      }
      if (asz != packed || st.n_red != sum_r || st.n_skel != sum_s || sum_r > n3)
        io_fail("corrupt factor file: phase sizes");
      for (int b = 0; b < nb; ++b) {
        const long long r = st.blocks[b].r(), s = st.blocks[b].s();
        const bool ok = st.o_a22[b] >= 0 && st.o_inv[b] >= 0 && st.o_x[b] >= 0 &&
                        st.o_w[b] >= 0 && st.o_red[b] >= 0 && st.o_skel[b] >= 0 &&
                        st.o_red[b] + r <= st.n_red && st.o_skel[b] + s <= st.n_skel;
        if (!ok) io_fail("corrupt factor file: block offsets");
      }
      if (step_arena_doubles(st) > asz) io_fail("corrupt factor file: block outside its arena");
      std::vector<int> red_all((size_t)st.n_red), skel_all((size_t)st.n_skel);
      rd.raw(red_all.data(), red_all.size() * sizeof(int));
      rd.raw(skel_all.data(), skel_all.size() * sizeof(int));
      for (const std::vector<int>* v : {&red_all, &skel_all})
        for (int g : *v)
          if (g < 0 || g >= n3) io_fail("corrupt factor file: DOF id out of range");
      st.arena = e.arena_factor.alloc<double>(asz);
      st.d_red = e.arena_factor.upload(red_all, e.stream);
      st.d_skel = e.arena_factor.upload(skel_all, e.stream);
      rd.device(st.arena, asz, e.stream);
      e.steps.push_back(std::move(st));
    }
    if (has_op) {
      op_touched = true;
      rd.device(e.d_band, 7 * n3, e.stream);
    }
    rd.finish();
    e.factor_precision = factor_precision;
    if (has_op) {
      // the operator and its symmetry (which elimination a refactorization uses)
      // travel together; without an operator in the file the handle keeps its own
      e.have_op = true;
      e.symmetric = symmetric;
    }
  } catch (...) {
    e.sync_quiet();
    e.release_factor();
    if (op_touched) e.have_op = false;  // the bands were partly overwritten
    throw;
  }
  e.factored = true;
  e.ensure_workspace(1);  // the apply sweeps of the loaded factor
  e.sync();
}
