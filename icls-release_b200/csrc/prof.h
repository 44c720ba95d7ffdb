// prof.h — per-launcher device timing on the context's stream.
//
// Every launcher opens a Scope named for its kernel(s): the scope counts the
// launches and, while profiling is on, brackets them with CUDA events on the
// context stream.  Elapsed times are folded in at the next read, after the
// stream has been synchronised.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace icls {

struct ProfEntry {
  std::string name;
  double total_ms = 0.0;
  long long launches = 0;  // kernel launches issued under this name
  long long timed = 0;     // launches bracketed by events
};

struct Prof {
  bool on = false;
  long long launches = 0;
  std::vector<ProfEntry> table;
  struct Pending { int id; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> pool;

  int id_of(const char* name) {
    for (size_t i = 0; i < table.size(); ++i)
      if (table[i].name == name) return (int)i;
    table.push_back(ProfEntry{name});
    return (int)table.size() - 1;
  }
  cudaEvent_t get() {
    if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  // fold completed events into the table (the caller synchronised the stream)
  void collect() {
    for (auto& p : pending) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
        table[p.id].total_ms += ms;
        table[p.id].timed += 1;
      }
      pool.push_back(p.a);
      pool.push_back(p.b);
    }
    pending.clear();
  }
  void release() {
    collect();
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
  }
};

class Scope {
 public:
  Scope(Prof& p, cudaStream_t s, const char* name, int nkernels = 1) : p_(p), s_(s) {
    id_ = p_.id_of(name);
    p_.table[id_].launches += nkernels;
    p_.launches += nkernels;
    if (p_.on) {
      a_ = p_.get();
      cudaEventRecord(a_, s_);
    }
  }
  ~Scope() {
    if (p_.on) {
      cudaEvent_t b = p_.get();
      cudaEventRecord(b, s_);
      p_.pending.push_back(Prof::Pending{id_, a_, b});
    }
  }

 private:
  Prof& p_;
  cudaStream_t s_;
  int id_ = 0;
  cudaEvent_t a_ = nullptr;
};

}  // namespace icls
