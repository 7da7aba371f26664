// Test-only: hera_b200/csrc/hera_combine.h driven by host threads with a
// fake batch function.  Built and run by tests/test_combine.py.
#include "../hera_b200/csrc/hera_combine.h"

#include <atomic>
#include <chrono>
#include <cstdio>
#include <random>
#include <thread>

// Every thread makes `calls` requests of random kind and size; the batch
// function records, per request, how many batches ran it and checks that a
// batch holds one kind and stays within the budget (unless it is a single
// request).  Returns the number of violations.
extern "C" int combine_check(int threads, int calls, int64_t budget, int kinds, unsigned seed,
			     unsigned long long *batches_out, unsigned long long *max_batch_out)
{
	hcomb::Combiner comb(budget);
	std::atomic<int> bad{0}, running{0};
	std::atomic<unsigned long long> max_batch{0};
	std::vector<std::thread> th;
	for (int t = 0; t < threads; ++t) {
		th.emplace_back([&, t] {
			std::mt19937 rng(seed + (unsigned)t);
			for (int c = 0; c < calls; ++c) {
				hcomb::Request r;
				r.kind = (int)(rng() % (unsigned)kinds);
				r.items = 1 + (int64_t)(rng() % 5000);
				int runs = 0;
				r.user = &runs;
				const int want = t * 100000 + c;
				int rc = comb.call(r, [&](std::vector<hcomb::Request *> &batch) {
					if (running.fetch_add(1) != 0)
						++bad;   // two batches at once
					int64_t items = 0;
					for (hcomb::Request *x : batch) {
						if (x->kind != batch[0]->kind)
							++bad;
						items += x->items;
						++*static_cast<int *>(x->user);
					}
					if (batch.size() > 1 && items > budget)
						++bad;
					unsigned long long n = batch.size(), m = max_batch.load();
					while (n > m && !max_batch.compare_exchange_weak(m, n))
						;
					std::this_thread::sleep_for(std::chrono::microseconds(50 + rng() % 200));
					for (hcomb::Request *x : batch)
						x->rc = x->kind * 7 + 1;
					running.fetch_sub(1);
				});
				if (runs != 1 || rc != r.kind * 7 + 1 || !r.done)
					++bad;
				(void)want;
			}
		});
	}
	for (auto &x : th)
		x.join();
	*batches_out = comb.batches();
	*max_batch_out = max_batch.load();
	return bad.load();
}
