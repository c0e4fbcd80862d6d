// Serving runtime: requests to factor a matrix and solve right-hand sides,
// admitted against an HBM budget, overlapped on one GPU.
//
//   submit     any host thread queues a request and returns; new
//              factorisations are charged their factor memory plus solve
//              scratch, follow-up solves their scratch, and a request is
//              admitted (first come first served, later requests may pass one
//              that does not fit yet) as soon as the budget has room
//   small      orders <= small_max_n: one worker thread takes every admitted
//              small request at once, packs the matrices into one buffer,
//              factors them in ONE persistent batched launch (batched.cu),
//              then solves, refines and measures all of them with batched
//              kernels (serve_kernels.cu) - requests that arrive meanwhile
//              form the next launch
//   large      larger orders: large_workers threads, each with its own
//              stream, run the blocked factorisation (mixed or plain) and the
//              refined solve (solve.cu) - several requests in flight overlap
//              on the device
//   resident   a factorisation with follow-up solves stays on the device
//              until its last follow-up is done; a stalled refinement on
//              mixed factors re-factors in FP64 and the factors stay FP64
// All device memory comes from the stream-ordered pool (cudaMallocAsync), so
// no allocation or release synchronises the device under concurrent work.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "delayed_pivoting_b200.h"
#include "dp_kernels.h"
#include "serve_kernels.h"

namespace {

using dp::Factor;
namespace sv = dp::serve;

double clock_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// One batched launch's factors in one pool block.
struct Group {
  char* mem = nullptr;
  double* base = nullptr;
  int *ipiv = nullptr, *jpiv = nullptr, *info = nullptr, *row = nullptr, *col = nullptr;
  std::vector<int> ns;
  std::vector<long long> off, rec;
  int live = 0;  // residents still using the factors (guarded by the server lock)
};

struct Resident {
  unsigned long long id = 0;
  int n = 0, lda = 0, small = 0;
  int left = 0;        // follow-ups still to complete
  int admits_left = 0; // follow-ups still to admit (extra ones are refused)
  const double* A = nullptr;
  Factor* factor = nullptr;          // large
  std::shared_ptr<Group> group;      // small
  int index = -1;
  size_t bytes = 0;                  // factor memory charged to the budget
  std::mutex m;                      // one solve at a time on `factor`
};

struct Job {
  dp_request r{};
  double t_submit = 0, t_admit = 0;
  size_t scratch = 0, factor = 0;    // charged bytes
  std::shared_ptr<Resident> res;     // follow-ups
};

size_t scratch_bytes(int n, int nrhs) {  // X, R, T of one solve, its columns in a coalesced solve
  return 4 * sizeof(double) * (size_t)n * nrhs + 4096;
}

size_t small_factor_bytes(int n) {
  return sizeof(double) * round_up((size_t)n * n, 4) + 5 * sizeof(int) * (size_t)n + 64;
}

size_t large_factor_bytes(int n) {
  // factors + composite orders, the blocked factorisation's workspace
  // (mailboxes, candidate rows, the BF16 pieces of the mixed updates: three
  // pieces of 256 columns for n + n and n + 256 operand rows; the outer
  // blocks' inverses and the 256-row copies of their block solves)
  return dp::factor_bytes(n) + 7168 * (size_t)n + (10u << 20);
}

}  // namespace

struct dp_server {
  dp_server_options opt{};
  int device = 0, sms = 0;
  size_t budget = 0;
  std::mutex m;
  std::condition_variable cv_large, cv_small, cv_done, cv_idle;
  std::deque<Job> pending, large_q, small_q;
  std::unordered_map<unsigned long long, std::shared_ptr<Resident>> residents;
  std::unordered_set<unsigned long long> live_ids;  // factorisations queued / running / resident
  std::vector<dp_request_result> done;
  size_t used = 0, peak = 0;
  bool stop = false;
  long long submitted = 0, completed = 0, small_launches = 0, small_items = 0, large_items = 0;
  int running = 0;
  std::vector<std::thread> threads;

  bool is_small(int n) const { return opt.small_max_n > 0 && n <= opt.small_max_n; }

  void charge(size_t b) {
    used += b;
    peak = std::max(peak, used);
  }
  void release(size_t b) { used -= std::min(used, b); }

  void finish_locked(const Job& j, dp_request_result r) {
    r.id = j.r.id;
    r.t_submit = j.t_submit;
    r.t_admit = j.t_admit;
    if (r.t_done == 0) r.t_done = clock_s();
    done.push_back(r);
    ++completed;
    cv_done.notify_all();
    cv_idle.notify_all();
  }

  // Admit what fits, in arrival order (called with the lock held).
  void schedule_locked() {
    bool to_small = false, to_large = false;
    for (auto it = pending.begin(); it != pending.end();) {
      Job& j = *it;
      if (j.r.factor_id != 0) {
        auto rit = residents.find(j.r.factor_id);
        if (rit == residents.end()) {
          if (live_ids.count(j.r.factor_id)) {  // its factorisation has not finished yet
            ++it;
            continue;
          }
          dp_request_result r{};
          r.status = DP_INVALID_ARGUMENT;
          r.info = -1;
          r.t_start = clock_s();
          finish_locked(j, r);
          it = pending.erase(it);
          continue;
        }
        if (rit->second->n != j.r.n || rit->second->admits_left <= 0) {
          dp_request_result r{};
          r.status = DP_INVALID_ARGUMENT;
          r.info = -1;
          finish_locked(j, r);
          it = pending.erase(it);
          continue;
        }
        j.res = rit->second;
      }
      const size_t need = j.scratch + j.factor;
      if (used + need > budget) {
        ++it;
        continue;
      }
      if (j.res) --j.res->admits_left;
      charge(need);
      j.t_admit = clock_s();
      if (is_small(j.r.n)) {
        small_q.push_back(j);
        to_small = true;
      } else {
        large_q.push_back(j);
        to_large = true;
      }
      it = pending.erase(it);
    }
    if (to_small) cv_small.notify_one();
    if (to_large) cv_large.notify_all();
  }

  void large_worker();
  void take_followups_locked(unsigned long long factor_id, int& rhs, std::vector<Job>& batch);
  void solve_large(std::vector<Job>& batch, size_t first, Factor* f, const double* A, int lda,
                   std::vector<dp_request_result>& out, cudaStream_t st);
  void small_worker();
  void run_small_new(std::vector<Job>& jobs, cudaStream_t st);
  void run_small_followups(std::vector<Job>& jobs, cudaStream_t st);
  void solve_refine(std::vector<sv::SolveItem>& items, std::vector<const Job*>& jobs,
                    std::vector<const double*>& As, std::vector<int>& ldas,
                    std::vector<dp_request_result>& out, cudaStream_t st);
  void drop_resident_locked(const std::shared_ptr<Resident>& r, cudaStream_t st);
};

void dp_server::drop_resident_locked(const std::shared_ptr<Resident>& r, cudaStream_t st) {
  release(r->bytes);
  residents.erase(r->id);
  live_ids.erase(r->id);
  if (r->factor) {
    dp::factor_destroy(r->factor, st);
    r->factor = nullptr;
  }
  if (r->group && --r->group->live == 0 && r->group->mem) {
    cudaFreeAsync(r->group->mem, st);
    r->group->mem = nullptr;
  }
  r->group.reset();
}

// Moves the admitted follow-up solves of factorisation `factor_id` out of
// the large queue into `batch` while the right-hand sides fit one solve
// (at most dp::serve::kMaxRhs columns in all).
void dp_server::take_followups_locked(unsigned long long factor_id, int& rhs,
                                      std::vector<Job>& batch) {
  for (auto it = large_q.begin(); it != large_q.end();) {
    if (it->r.factor_id == factor_id && rhs + it->r.nrhs <= dp::serve::kMaxRhs) {
      rhs += it->r.nrhs;
      batch.push_back(*it);
      ++running;
      it = large_q.erase(it);
    } else {
      ++it;
    }
  }
}

// Solves batch[first..] with the factors f in ONE refined multi-RHS solve:
// the requests' right-hand sides are copied side by side into one n x k
// block (k = sum of their nrhs), solved together, and the solution columns
// copied back; one request is solved in place.  Every request gets the
// combined solve's backward error (the largest over all columns) and
// refinement steps, and its share of the device time.
void dp_server::solve_large(std::vector<Job>& batch, size_t first, Factor* f, const double* A,
                            int lda, std::vector<dp_request_result>& out, cudaStream_t st) {
  const int n = f->n;
  const size_t cnt = batch.size() - first;
  if (cnt == 0) return;
  int k = 0;
  for (size_t i = first; i < batch.size(); ++i) k += batch[i].r.nrhs;
  dp_ir_result ir{};
  int status = DP_SUCCESS;
  double* W = nullptr;
  if (cnt == 1) {
    const Job& j = batch[first];
    status = dp::factor_solve(f, A, lda, j.r.d_b, j.r.ldb, j.r.nrhs, opt.max_iter, opt.tol, &ir, st);
  } else {
    if (cudaMallocAsync(reinterpret_cast<void**>(&W), sizeof(double) * (size_t)n * k, st) !=
        cudaSuccess) {
      cudaGetLastError();
      W = nullptr;
      status = DP_ALLOCATION_FAILED;
    }
    int c = 0;
    for (size_t i = first; i < batch.size() && status == DP_SUCCESS; ++i) {
      const Job& j = batch[i];
      if (cudaMemcpy2DAsync(W + (size_t)c * n, sizeof(double) * n, j.r.d_b,
                            sizeof(double) * j.r.ldb, sizeof(double) * n, j.r.nrhs,
                            cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        status = DP_CUDA_FAILURE;
      c += j.r.nrhs;
    }
    if (status == DP_SUCCESS)
      status = dp::factor_solve(f, A, lda, W, n, k, opt.max_iter, opt.tol, &ir, st);
    c = 0;
    for (size_t i = first; i < batch.size() && status == DP_SUCCESS; ++i) {
      const Job& j = batch[i];
      if (cudaMemcpy2DAsync(j.r.d_b, sizeof(double) * j.r.ldb, W + (size_t)c * n,
                            sizeof(double) * n, sizeof(double) * n, j.r.nrhs,
                            cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        status = DP_CUDA_FAILURE;
      c += j.r.nrhs;
    }
    if (W) cudaFreeAsync(W, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && status == DP_SUCCESS) status = DP_CUDA_FAILURE;
  }
  const double solve_ms = ir.total_ms - ir.factor_ms;
  for (size_t i = first; i < batch.size(); ++i) {
    dp_request_result& r = out[i];
    r.status = status;
    r.info = f->info;
    r.precision = f->precision;
    r.iterations = ir.iterations;
    r.refactored = ir.refactored;
    r.backward_error = ir.backward_error;
    r.factor_ms += i == first ? ir.factor_ms : 0.0;
    r.solve_ms = solve_ms * batch[i].r.nrhs / (double)k;
  }
}

void dp_server::large_worker() {
  cudaSetDevice(device);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (;;) {
    std::vector<Job> batch;  // batch[0] as popped; then follow-ups of the same factorisation
    int rhs = 0;
    {
      std::unique_lock<std::mutex> lk(m);
      cv_large.wait(lk, [&] { return stop || !large_q.empty(); });
      if (large_q.empty()) break;
      batch.push_back(large_q.front());
      large_q.pop_front();
      ++running;
      rhs = batch[0].r.nrhs;
      if (batch[0].r.factor_id != 0) take_followups_locked(batch[0].r.factor_id, rhs, batch);
    }
    std::vector<dp_request_result> out(batch.size());
    for (auto& r : out) {
      r.path = 1;
      r.t_start = clock_s();
    }
    // copies: appending follow-ups to `batch` may move its elements
    const dp_request r0 = batch[0].r;
    const size_t factor0 = batch[0].factor;
    const std::shared_ptr<Resident> res0 = batch[0].res;
    std::shared_ptr<Resident> keep;
    if (r0.factor_id == 0) {
      Factor* f = nullptr;
      // mixed factors only from mixed_min_n up, where they are faster than FP64
      const int prec = opt.mixed_min_n < 0 || r0.n >= opt.mixed_min_n ? opt.precision
                                                                       : DP_PRECISION_FP64;
      const int status = dp::factor_create(&f, r0.n, r0.d_a, r0.lda, prec, st, opt.panel_rows);
      out[0].status = status;
      out[0].info = f ? f->info : -1;
      if (f) out[0].factor_ms = f->factor_ms;
      if (status == DP_SUCCESS && r0.followups > 0 && f && f->info == r0.n) {
        keep = std::make_shared<Resident>();
        keep->id = r0.id;
        keep->n = r0.n;
        keep->lda = r0.lda;
        keep->A = r0.d_a;
        keep->factor = f;
        keep->left = keep->admits_left = r0.followups;
        keep->bytes = factor0;
        // resident before the first solve: follow-ups already submitted are
        // admitted now and solved together with it
        std::lock_guard<std::mutex> lk(m);
        residents[keep->id] = keep;
        schedule_locked();
        take_followups_locked(keep->id, rhs, batch);
        out.resize(batch.size());
        for (size_t i = 1; i < out.size(); ++i) {
          out[i].path = 1;
          out[i].t_start = clock_s();
        }
      }
      if (status == DP_SUCCESS) {
        std::unique_lock<std::mutex> g;
        if (keep) g = std::unique_lock<std::mutex>(keep->m);
        solve_large(batch, 0, f, r0.d_a, r0.lda, out, st);
      }
      if (!keep && f) dp::factor_destroy(f, st);
    } else {
      std::lock_guard<std::mutex> g(res0->m);
      solve_large(batch, 0, res0->factor, res0->A, res0->lda, out, st);
    }
    const double t_done = clock_s();
    {
      std::lock_guard<std::mutex> lk(m);
      for (size_t i = 0; i < batch.size(); ++i) {
        Job& b = batch[i];
        dp_request_result r = out[i];
        r.t_done = t_done;
        release(b.scratch);
        if (b.r.factor_id == 0) {
          if (!keep) {
            release(b.factor);
            live_ids.erase(b.r.id);
          }
        } else if (--b.res->left == 0) {
          drop_resident_locked(b.res, st);
        }
        ++large_items;
        --running;
        finish_locked(b, r);
      }
      schedule_locked();
    }
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
}

// X = A^{-1} B with FP64 refinement for every item: items[i] solves with
// jobs[i]'s right-hand sides into scratch X, the corrections come from the
// same factors, and the refined X is copied into the caller's B.
void dp_server::solve_refine(std::vector<sv::SolveItem>& items, std::vector<const Job*>& jobs,
                             std::vector<const double*>& As, std::vector<int>& ldas,
                             std::vector<dp_request_result>& out, cudaStream_t st) {
  const int k = (int)items.size();
  if (k == 0) return;
  size_t xs = 0;
  std::vector<size_t> xoff(k);
  int max_n = 1;
  for (int i = 0; i < k; ++i) {
    xoff[i] = xs;
    xs += round_up((size_t)items[i].n * items[i].nrhs, 4);
    max_n = std::max(max_n, items[i].n);
  }
  const size_t item_bytes =
      round_up(sizeof(sv::SolveItem) * k, 256) + round_up(sizeof(sv::ResidualItem) * k, 256) +
      round_up(sizeof(sv::AxpyItem) * k, 256) + round_up(sizeof(sv::CopyItem) * k, 256) +
      round_up(sizeof(double) * k, 256);
  char* mem = nullptr;
  const size_t bytes = 3 * sizeof(double) * xs + item_bytes;
  auto fail = [&](int status) {
    for (int i = 0; i < k; ++i) out[i].status = status;
  };
  if (cudaMallocAsync(reinterpret_cast<void**>(&mem), bytes, st) != cudaSuccess) {
    cudaGetLastError();
    return fail(DP_ALLOCATION_FAILED);
  }
  double* X = reinterpret_cast<double*>(mem);
  double* R = X + xs;
  double* D = R + xs;
  char* p = reinterpret_cast<char*>(D + xs);
  auto* d_solve = reinterpret_cast<sv::SolveItem*>(p);
  p += round_up(sizeof(sv::SolveItem) * k, 256);
  auto* d_res = reinterpret_cast<sv::ResidualItem*>(p);
  p += round_up(sizeof(sv::ResidualItem) * k, 256);
  auto* d_axpy = reinterpret_cast<sv::AxpyItem*>(p);
  p += round_up(sizeof(sv::AxpyItem) * k, 256);
  auto* d_copy = reinterpret_cast<sv::CopyItem*>(p);
  p += round_up(sizeof(sv::CopyItem) * k, 256);
  auto* d_err = reinterpret_cast<double*>(p);

  int status = DP_SUCCESS;
  auto upload = [&](void* dst, const void* src, size_t n) {
    if (status == DP_SUCCESS &&
        cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) != cudaSuccess)
      status = DP_CUDA_FAILURE;
  };
  auto ok = [&](int s) {
    if (status == DP_SUCCESS && s != DP_SUCCESS) status = s;
  };
  // first solve: B -> X
  for (int i = 0; i < k; ++i) {
    items[i].X = X + xoff[i];
    items[i].ldx = items[i].n;
  }
  upload(d_solve, items.data(), sizeof(sv::SolveItem) * k);
  if (status == DP_SUCCESS) ok(sv::launch_solve(d_solve, k, max_n, st));

  std::vector<int> active(k);
  for (int i = 0; i < k; ++i) active[i] = i;
  std::vector<double> prev(k, INFINITY), err(k);
  for (int it = 0; status == DP_SUCCESS && !active.empty(); ++it) {
    const int a = (int)active.size();
    std::vector<sv::ResidualItem> ri(a);
    for (int q = 0; q < a; ++q) {
      const int i = active[q];
      ri[q] = sv::ResidualItem{As[i], jobs[i]->r.d_b, X + xoff[i], R + xoff[i], items[i].n,
                               items[i].nrhs, ldas[i], jobs[i]->r.ldb, items[i].n, items[i].n};
    }
    upload(d_res, ri.data(), sizeof(sv::ResidualItem) * a);
    if (status == DP_SUCCESS) ok(sv::launch_residual(d_res, d_err, a, max_n, st));
    if (status == DP_SUCCESS &&
        (cudaMemcpyAsync(err.data(), d_err, sizeof(double) * a, cudaMemcpyDeviceToHost, st) !=
             cudaSuccess ||
         cudaStreamSynchronize(st) != cudaSuccess))
      status = DP_CUDA_FAILURE;
    if (status != DP_SUCCESS) break;
    std::vector<int> next;
    for (int q = 0; q < a; ++q) {
      const int i = active[q];
      out[i].backward_error = err[q];
      if (err[q] <= opt.tol || it >= opt.max_iter || (it > 0 && !(err[q] <= 0.5 * prev[i])))
        continue;
      prev[i] = err[q];
      next.push_back(i);
    }
    if (next.empty()) break;
    // corrections D = A^{-1} R, X += D
    const int c = (int)next.size();
    std::vector<sv::SolveItem> si(c);
    std::vector<sv::AxpyItem> ai(c);
    for (int q = 0; q < c; ++q) {
      const int i = next[q];
      si[q] = items[i];
      si[q].B = R + xoff[i];
      si[q].ldb = items[i].n;
      si[q].X = D + xoff[i];
      si[q].ldx = items[i].n;
      ai[q] = sv::AxpyItem{X + xoff[i], D + xoff[i], items[i].n, items[i].nrhs, items[i].n,
                           items[i].n};
      out[i].iterations += 1;
    }
    upload(d_solve, si.data(), sizeof(sv::SolveItem) * c);
    if (status == DP_SUCCESS) ok(sv::launch_solve(d_solve, c, max_n, st));
    upload(d_axpy, ai.data(), sizeof(sv::AxpyItem) * c);
    if (status == DP_SUCCESS) ok(sv::launch_axpy(d_axpy, c, st));
    active.swap(next);
  }
  // X -> B
  std::vector<sv::CopyItem> ci(k);
  for (int i = 0; i < k; ++i)
    ci[i] = sv::CopyItem{jobs[i]->r.d_b, X + xoff[i], items[i].n, items[i].nrhs, jobs[i]->r.ldb,
                         items[i].n};
  upload(d_copy, ci.data(), sizeof(sv::CopyItem) * k);
  if (status == DP_SUCCESS) ok(sv::launch_copy(d_copy, k, st));
  if (cudaStreamSynchronize(st) != cudaSuccess && status == DP_SUCCESS) status = DP_CUDA_FAILURE;
  cudaFreeAsync(mem, st);
  if (status != DP_SUCCESS) fail(status);
}

void dp_server::run_small_new(std::vector<Job>& jobs, cudaStream_t st) {
  const int k = (int)jobs.size();
  auto g = std::make_shared<Group>();
  g->ns.resize(k);
  g->off.resize(k);
  g->rec.resize(k);
  long long elems = 0, recs = 0;
  int max_n = 1;
  for (int i = 0; i < k; ++i) {
    const int n = jobs[i].r.n;
    g->ns[i] = n;
    g->off[i] = elems;
    g->rec[i] = recs;
    elems += ((long long)n * n + 3) & ~3LL;
    recs += n;
    max_n = std::max(max_n, n);
  }
  std::vector<int> order(k);
  for (int i = 0; i < k; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return g->ns[a] > g->ns[b]; });
  // one pool block: factors, records, orders, info | metadata | packing items
  const size_t b_base = sizeof(double) * (size_t)elems;
  const size_t b_recs = round_up(sizeof(int) * (size_t)recs, 256);
  const size_t b_cnt = round_up(sizeof(int) * (size_t)k, 256);
  const size_t b_ll = round_up(sizeof(long long) * (size_t)k, 256);
  const size_t b_copy = round_up(sizeof(sv::CopyItem) * (size_t)k, 256);
  const size_t total = round_up(b_base, 256) + 4 * b_recs + 3 * b_cnt + 2 * b_ll + 256 + b_copy;
  std::vector<dp_request_result> out(k);
  for (auto& r : out) {
    r.path = 0;
    r.precision = DP_PRECISION_FP64;
    r.t_start = clock_s();
    r.info = -1;
  }
  int status = DP_SUCCESS;
  if (cudaMallocAsync(reinterpret_cast<void**>(&g->mem), total, st) != cudaSuccess) {
    cudaGetLastError();
    g->mem = nullptr;
    status = DP_ALLOCATION_FAILED;
  }
  std::vector<int> info(k, -1);
  if (status == DP_SUCCESS) {
    char* p = g->mem;
    g->base = reinterpret_cast<double*>(p);
    p += round_up(b_base, 256);
    g->ipiv = reinterpret_cast<int*>(p);
    p += b_recs;
    g->jpiv = reinterpret_cast<int*>(p);
    p += b_recs;
    g->row = reinterpret_cast<int*>(p);
    p += b_recs;
    g->col = reinterpret_cast<int*>(p);
    p += b_recs;
    g->info = reinterpret_cast<int*>(p);
    p += b_cnt;
    int* d_n = reinterpret_cast<int*>(p);
    p += b_cnt;
    int* d_order = reinterpret_cast<int*>(p);
    p += b_cnt;
    long long* d_off = reinterpret_cast<long long*>(p);
    p += b_ll;
    long long* d_rec = reinterpret_cast<long long*>(p);
    p += b_ll;
    int* d_queue = reinterpret_cast<int*>(p);
    p += 256;
    auto* d_copy = reinterpret_cast<sv::CopyItem*>(p);
    std::vector<sv::CopyItem> ci(k);
    for (int i = 0; i < k; ++i)
      ci[i] = sv::CopyItem{g->base + g->off[i], jobs[i].r.d_a, g->ns[i], g->ns[i], g->ns[i],
                           jobs[i].r.lda};
    auto up = [&](void* dst, const void* src, size_t n) {
      if (status == DP_SUCCESS &&
          cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st) != cudaSuccess)
        status = DP_CUDA_FAILURE;
    };
    up(d_n, g->ns.data(), sizeof(int) * k);
    up(d_order, order.data(), sizeof(int) * k);
    up(d_off, g->off.data(), sizeof(long long) * k);
    up(d_rec, g->rec.data(), sizeof(long long) * k);
    up(d_copy, ci.data(), sizeof(sv::CopyItem) * k);
    if (status == DP_SUCCESS) status = sv::launch_copy(d_copy, k, st);
    dp_batch_options bo;
    dp_batch_options_init(&bo);
    if (status == DP_SUCCESS)
      status = dp::batch::launch_raw(k, max_n, sms, d_n, d_off, d_rec, d_order, d_queue, g->base,
                                     g->ipiv, g->jpiv, g->info, bo, st);
    if (status == DP_SUCCESS)
      status = sv::launch_orders(d_n, d_rec, g->ipiv, g->jpiv, g->row, g->col, k, st);
    if (status == DP_SUCCESS &&
        (cudaMemcpyAsync(info.data(), g->info, sizeof(int) * k, cudaMemcpyDeviceToHost, st) !=
             cudaSuccess ||
         cudaStreamSynchronize(st) != cudaSuccess))
      status = DP_CUDA_FAILURE;
  }
  std::vector<sv::SolveItem> items;
  std::vector<const Job*> sj;
  std::vector<const double*> As;
  std::vector<int> ldas, map;
  std::vector<dp_request_result> sub;
  for (int i = 0; i < k; ++i) {
    out[i].status = status;
    out[i].info = status == DP_SUCCESS ? info[i] : -1;
    if (status != DP_SUCCESS || info[i] < g->ns[i]) continue;
    items.push_back(sv::SolveItem{g->base + g->off[i], g->row + g->rec[i], g->col + g->rec[i],
                                  jobs[i].r.d_b, nullptr, g->ns[i], jobs[i].r.nrhs, jobs[i].r.ldb,
                                  0});
    sj.push_back(&jobs[i]);
    As.push_back(jobs[i].r.d_a);
    ldas.push_back(jobs[i].r.lda);
    map.push_back(i);
    sub.push_back(out[i]);
  }
  solve_refine(items, sj, As, ldas, sub, st);
  for (size_t q = 0; q < map.size(); ++q) out[map[q]] = sub[q];
  const double t = clock_s();
  std::lock_guard<std::mutex> lk(m);
  ++small_launches;
  for (int i = 0; i < k; ++i) {
    Job& j = jobs[i];
    release(j.scratch);
    if (out[i].status == DP_SUCCESS && j.r.followups > 0 && out[i].info == j.r.n) {
      auto res = std::make_shared<Resident>();
      res->id = j.r.id;
      res->n = j.r.n;
      res->lda = j.r.lda;
      res->A = j.r.d_a;
      res->small = 1;
      res->group = g;
      res->index = i;
      res->left = res->admits_left = j.r.followups;
      res->bytes = j.factor;
      ++g->live;
      residents[res->id] = res;
    } else {
      release(j.factor);
      live_ids.erase(j.r.id);
    }
    out[i].t_done = t;
    ++small_items;
    finish_locked(j, out[i]);
  }
  if (g->live == 0 && g->mem) {
    cudaFreeAsync(g->mem, st);
    g->mem = nullptr;
  }
  running -= k;
  schedule_locked();
}

void dp_server::run_small_followups(std::vector<Job>& jobs, cudaStream_t st) {
  const int k = (int)jobs.size();
  std::vector<dp_request_result> out(k);
  std::vector<sv::SolveItem> items(k);
  std::vector<const Job*> sj(k);
  std::vector<const double*> As(k);
  std::vector<int> ldas(k);
  for (int i = 0; i < k; ++i) {
    const Resident& r = *jobs[i].res;
    const Group& g = *r.group;
    out[i].path = 0;
    out[i].precision = DP_PRECISION_FP64;
    out[i].info = r.n;
    out[i].t_start = clock_s();
    items[i] = sv::SolveItem{g.base + g.off[r.index], g.row + g.rec[r.index],
                             g.col + g.rec[r.index], jobs[i].r.d_b, nullptr, r.n, jobs[i].r.nrhs,
                             jobs[i].r.ldb, 0};
    sj[i] = &jobs[i];
    As[i] = r.A;
    ldas[i] = r.lda;
  }
  solve_refine(items, sj, As, ldas, out, st);
  const double t = clock_s();
  std::lock_guard<std::mutex> lk(m);
  for (int i = 0; i < k; ++i) {
    Job& j = jobs[i];
    release(j.scratch);
    if (--j.res->left == 0) drop_resident_locked(j.res, st);
    out[i].t_done = t;
    ++small_items;
    finish_locked(j, out[i]);
  }
  running -= k;
  schedule_locked();
}

void dp_server::small_worker() {
  cudaSetDevice(device);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (;;) {
    std::vector<Job> fresh, follow;
    {
      std::unique_lock<std::mutex> lk(m);
      cv_small.wait(lk, [&] { return stop || !small_q.empty(); });
      if (small_q.empty()) break;
      while (!small_q.empty() && (int)(fresh.size() + follow.size()) < opt.small_max_batch) {
        Job j = small_q.front();
        small_q.pop_front();
        (j.r.factor_id == 0 ? fresh : follow).push_back(j);
      }
      running += (int)(fresh.size() + follow.size());
    }
    if (!fresh.empty()) run_small_new(fresh, st);
    if (!follow.empty()) run_small_followups(follow, st);
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
}

// Default order from which a mixed server factors in mixed precision (the
// measured crossover of factor + refined solve against FP64 on B200).
constexpr int kMixedMinN = 12288;

extern "C" {

void dp_server_options_init(dp_server_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->budget_bytes = 160ull << 30;
  o->precision = DP_PRECISION_MIXED_BF16X6;
  o->large_workers = 6;
  o->small_max_n = DP_BATCH_MAX_N;
  o->small_max_batch = 2048;
  o->max_iter = 10;
  o->tol = 1e-14;
  o->mixed_min_n = kMixedMinN;
}

double dp_server_clock(void) { return clock_s(); }

int dp_server_create(dp_server** out, const dp_server_options* opt) {
  if (!out) return DP_INVALID_ARGUMENT;
  *out = nullptr;
  dp_server_options o;
  dp_server_options_init(&o);
  if (opt) {
    o = *opt;
    if (o.budget_bytes == 0) o.budget_bytes = 160ull << 30;
    if (o.small_max_n == 0) o.small_max_n = DP_BATCH_MAX_N;
    if (o.small_max_batch == 0) o.small_max_batch = 2048;
    if (o.max_iter == 0) o.max_iter = 10;
    if (o.tol == 0.0) o.tol = 1e-14;
    if (o.mixed_min_n == 0) o.mixed_min_n = kMixedMinN;
  }
  if (o.large_workers == 0) o.large_workers = 6;
  if (!dp::valid_precision(o.precision) ||
      o.large_workers < 1 || o.large_workers > 64 || o.small_max_n > DP_BATCH_MAX_N ||
      o.panel_rows < 0 || o.mixed_min_n < -1 ||
      o.small_max_batch < 1 || o.max_iter < 0 || !(o.tol > 0.0))
    return DP_INVALID_ARGUMENT;
  auto* s = new (std::nothrow) dp_server;
  if (!s) return DP_ALLOCATION_FAILED;
  s->opt = o;
  s->budget = (size_t)o.budget_bytes;
  if (cudaGetDevice(&s->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device) != cudaSuccess) {
    delete s;
    return DP_CUDA_FAILURE;
  }
  for (int i = 0; i < o.large_workers; ++i) s->threads.emplace_back([s] { s->large_worker(); });
  if (o.small_max_n > 0) s->threads.emplace_back([s] { s->small_worker(); });
  *out = s;
  return DP_SUCCESS;
}

int dp_server_submit(dp_server* s, const dp_request* q) {
  if (!s || !q) return DP_INVALID_ARGUMENT;
  const dp_request& r = *q;
  if (r.id == 0 || r.n < 1 || r.lda < r.n || r.ldb < r.n || r.nrhs < 1 ||
      r.nrhs > dp::serve::kMaxRhs || (!r.d_a && r.factor_id == 0) || !r.d_b || r.followups < 0 ||
      (r.factor_id != 0 && r.followups != 0))
    return DP_INVALID_ARGUMENT;
  Job j;
  j.r = r;
  j.t_submit = clock_s();
  j.scratch = scratch_bytes(r.n, r.nrhs);
  if (r.factor_id == 0)
    j.factor = s->is_small(r.n) ? small_factor_bytes(r.n) : large_factor_bytes(r.n);
  if (j.scratch + j.factor > s->budget) return DP_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->m);
  if (s->stop) return DP_INVALID_ARGUMENT;
  if (r.factor_id == 0) {
    if (s->live_ids.count(r.id)) return DP_INVALID_ARGUMENT;
    s->live_ids.insert(r.id);
  } else if (!s->live_ids.count(r.factor_id)) {
    return DP_INVALID_ARGUMENT;  // no such factorisation queued, running or resident
  }
  s->pending.push_back(j);
  ++s->submitted;
  s->schedule_locked();
  return DP_SUCCESS;
}

int dp_server_poll(dp_server* s, dp_request_result* out, int max, int wait_ms) {
  if (!s || !out || max < 1) return 0;
  std::unique_lock<std::mutex> lk(s->m);
  if (s->done.empty() && wait_ms > 0)
    s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
  const int k = std::min<int>(max, (int)s->done.size());
  std::copy(s->done.begin(), s->done.begin() + k, out);
  s->done.erase(s->done.begin(), s->done.begin() + k);
  return k;
}

int dp_server_stats_get(dp_server* s, dp_server_stats* o) {
  if (!s || !o) return DP_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->m);
  o->bytes_in_use = s->used;
  o->bytes_peak = s->peak;
  o->submitted = s->submitted;
  o->completed = s->completed;
  o->pending = (long long)(s->pending.size() + s->small_q.size() + s->large_q.size()) + s->running;
  o->residents = (long long)s->residents.size();
  o->small_launches = s->small_launches;
  o->small_items = s->small_items;
  o->large_items = s->large_items;
  return DP_SUCCESS;
}

void dp_server_destroy(dp_server* s) {
  if (!s) return;
  {
    // wait for every admitted or admissible request; follow-ups whose
    // factorisation never arrives are dropped
    std::unique_lock<std::mutex> lk(s->m);
    s->cv_idle.wait(lk, [&] {
      if (!s->small_q.empty() || !s->large_q.empty() || s->running > 0) return false;
      for (const Job& j : s->pending)
        if (j.scratch + j.factor + s->used <= s->budget) return false;
      return true;
    });
    s->stop = true;
  }
  s->cv_large.notify_all();
  s->cv_small.notify_all();
  for (auto& t : s->threads) t.join();
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  {
    std::lock_guard<std::mutex> lk(s->m);
    std::vector<std::shared_ptr<Resident>> all;
    for (auto& kv : s->residents) all.push_back(kv.second);
    for (auto& r : all) s->drop_resident_locked(r, st);
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  delete s;
}

}  // extern "C"
