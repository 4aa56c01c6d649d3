// Parallel text writers for the drop-in executables (host code, header-only).
//
// The upstream executables format every output with iostream: C and Viss with
// the default float format (printf "%g", 6 significant digits), the baseline
// tables with std::scientific and precision 15 (printf "%.15e")
// (main_recon_online.cu:358-362, 516-538; common.hpp:145-153).  Single-threaded
// iostream output of the 2e8-line C file of a 10 MHz run takes longer than
// the run itself.  Here rows are formatted with std::to_chars (defined as
// printf with the same conversion, so the bytes are identical) in parallel
// blocks and written in order; an AsyncWriter runs whole-file jobs on a
// background thread so that a day's files are written while the next day
// computes.
#pragma once

#include <algorithm>
#include <atomic>
#include <charconv>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace vbtext {

enum class Fmt { General6, Sci15 };

struct Col {
  const float* p;
  size_t stride;   // in floats
};

// Appends one value as printf("%g") / printf("%.15e") would print it.
inline void put_value(std::string& out, float v, Fmt fmt) {
  char buf[64];
  std::to_chars_result r = (fmt == Fmt::General6)
                               ? std::to_chars(buf, buf + sizeof(buf), (double)v, std::chars_format::general, 6)
                               : std::to_chars(buf, buf + sizeof(buf), (double)v, std::chars_format::scientific, 15);
  out.append(buf, r.ptr);
}

// Rows [r0, r1) as text: columns separated by one space, '\n' after each row.
inline void format_rows(std::string& out, const std::vector<Col>& cols, size_t r0, size_t r1, Fmt fmt) {
  out.clear();
  out.reserve((r1 - r0) * cols.size() * (fmt == Fmt::General6 ? 13 : 24));
  for (size_t r = r0; r < r1; ++r) {
    for (size_t c = 0; c < cols.size(); ++c) {
      if (c) out.push_back(' ');
      put_value(out, cols[c].p[r * cols[c].stride], fmt);
    }
    out.push_back('\n');
  }
}

// Writes `rows` rows of `cols` to `path`; blocks of rows are formatted in
// parallel (OpenMP when the translation unit is built with it) and written in
// order, a bounded number of blocks at a time.
inline bool write_rows(const std::string& path, const std::vector<Col>& cols, size_t rows, Fmt fmt) {
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const size_t block = 1 << 16;
  const size_t wave = 64;   // blocks formatted per round
  std::vector<std::string> bufs(wave);
  bool ok = true;
  for (size_t b0 = 0; b0 * block < rows && ok; b0 += wave) {
    const size_t nb = std::min(wave, (rows - b0 * block + block - 1) / block);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < (long long)nb; ++k) {
      const size_t r0 = (b0 + (size_t)k) * block;
      const size_t r1 = std::min(rows, r0 + block);
      format_rows(bufs[(size_t)k], cols, r0, r1, fmt);
    }
    for (size_t k = 0; k < nb && ok; ++k)
      ok = std::fwrite(bufs[k].data(), 1, bufs[k].size(), f) == bufs[k].size();
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

inline bool write_binary(const std::string& path, const void* data, size_t bytes) {
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(data, 1, bytes, f) == bytes;
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

// One background thread running file jobs in submission order.  A job owns
// its data (captured by value / move) and returns false on failure; wait()
// returns false if any job failed.  Jobs never print: they queue messages
// with log(), which the owning thread prints with drain() at points of its
// choosing, so that no output line is interleaved.
class AsyncWriter {
 public:
  void log(std::string msg) {
    std::lock_guard<std::mutex> lk(log_mu_);
    logs_.push_back(std::move(msg));
  }
  template <class Stream>
  void drain(Stream& os) {
    std::deque<std::string> l;
    {
      std::lock_guard<std::mutex> lk(log_mu_);
      l.swap(logs_);
    }
    for (auto& m : l) os << m;
  }
  explicit AsyncWriter(bool enabled) : enabled_(enabled) {
    if (enabled_) th_ = std::thread([this] { loop(); });
  }
  ~AsyncWriter() { wait(); }
  void submit(std::function<bool()> job) {
    if (!enabled_) {
      if (!job()) failed_ = true;
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(std::move(job));
    }
    cv_.notify_one();
  }
  bool wait() {
    if (enabled_ && th_.joinable()) {
      {
        std::lock_guard<std::mutex> lk(mu_);
        done_ = true;
      }
      cv_.notify_one();
      th_.join();
    }
    return !failed_;
  }

 private:
  void loop() {
    for (;;) {
      std::function<bool()> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return done_ || !q_.empty(); });
        if (q_.empty()) return;
        job = std::move(q_.front());
        q_.pop_front();
      }
      if (!job()) failed_ = true;
    }
  }
  bool enabled_;
  bool done_ = false;
  std::atomic<bool> failed_{false};
  std::mutex log_mu_;
  std::deque<std::string> logs_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<std::function<bool()>> q_;
  std::thread th_;
};

}  // namespace vbtext
