// hera_combine.h -- host-side combining of concurrent calls on one context.
//
// hera's paired-end workers (align_pool_pair, src/hash_align.c:1855-1946)
// each parse a 1 MB buffer pair (src/get_buffer.c:3), about 4,500 read
// pairs, and align it.  One device call for so few pairs is mostly fixed
// cost, so the drop-in entries combine the calls that several worker
// threads make at the same time on one context: a caller queues its
// request; if no call is running, it becomes the leader, takes every queued
// request that can share a device batch with the first (same kind, up to a
// pair budget) and runs them as one batch; the others wait until their
// request is done.  A request left queued when a batch ends is taken by the
// next leader, which is one of the waiting callers.  No timers: batches
// grow by themselves while the device is busy.
//
// Host-only C++ (no CUDA): tests/combine_check.cpp drives it with threads.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <vector>

namespace hcomb {

struct Request {
	int kind = 0;         // requests of one kind only share a batch
	int64_t items = 0;    // its size against the batch budget
	int rc = 0;           // set by the batch
	bool done = false;
	void *user = nullptr;
};

class Combiner {
public:
	explicit Combiner(int64_t budget) : budget_(budget) {}

	// Queue `r`, and run batches (as leader) or wait until `r` is done.
	// `run(batch)` runs one batch (called without the lock held) and sets
	// each request's rc.
	template <class Run>
	int call(Request &r, Run run)
	{
		std::unique_lock<std::mutex> lk(mu_);
		q_.push_back(&r);
		while (!r.done) {
			if (leader_) {
				cv_.wait(lk);
				continue;
			}
			leader_ = true;
			std::vector<Request *> batch = take();
			++batches_;
			lk.unlock();
			run(batch);
			lk.lock();
			for (Request *x : batch)
				x->done = true;
			leader_ = false;
			cv_.notify_all();
		}
		return r.rc;
	}

	uint64_t batches() const
	{
		std::lock_guard<std::mutex> g(mu_);
		return batches_;
	}

private:
	// the first queued request and every later one of its kind that fits
	// the budget (the first is always taken, whatever its size)
	std::vector<Request *> take()
	{
		std::vector<Request *> batch, rest;
		int64_t items = 0;
		const int kind = q_.front()->kind;
		for (Request *x : q_) {
			if (x->kind == kind && (batch.empty() || items + x->items <= budget_)) {
				batch.push_back(x);
				items += x->items;
			} else {
				rest.push_back(x);
			}
		}
		q_.swap(rest);
		return batch;
	}

	mutable std::mutex mu_;
	std::condition_variable cv_;
	std::vector<Request *> q_;
	bool leader_ = false;
	uint64_t batches_ = 0;
	int64_t budget_;
};

}   // namespace hcomb
