// Multi-process shared-memory implementation of the MPI subset declared in mpi.h (test
// infrastructure: it runs the reference's multi-rank CPU path on one machine).  See mpi.h.
#include "mpi.h"

#include <sched.h>
#include <signal.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

constexpr int kMaxRanks = 64;
constexpr size_t kSlot = 64 * 1024;       // collective payload per rank
constexpr size_t kChunk = 512 * 1024;     // channel chunk

struct Channel {
	alignas(64) std::atomic<int> full;      // 1: a chunk of `len` bytes is waiting
	size_t len;
	char data[kChunk];
};

struct Shared {
	alignas(64) std::atomic<int> bar_count;
	alignas(64) std::atomic<int> bar_phase;
	alignas(64) std::atomic<int> failed;      // a rank gave up waiting
	alignas(64) char slot[kMaxRanks][kSlot];
	Channel chan[1];                          // [src * size + dst], size * size of them
};

Shared *g_sh = nullptr;
int g_rank = 0, g_size = 1;
int g_phase = 0;
std::vector<pid_t> g_children;
double g_timeout = 900.0;

double now() {
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

// Spin (then yield) until ready() holds; abort the process group after g_timeout seconds or when
// another rank has given up.
template<typename F>
void wait_until(F ready, const char *what) {
	double t0 = 0.0;
	for (long it = 0;; it++) {
		if (ready()) return;
		if (it < 2000) continue;
		sched_yield();
		if ((it & 1023) == 0) {
			if (t0 == 0.0) t0 = now();
			if (g_sh->failed.load() || now() - t0 > g_timeout) {
				g_sh->failed.store(1);
				std::fprintf(stderr, "mpi_shm: rank %d gave up waiting in %s\n", g_rank, what);
				std::fflush(stderr);
				kill(0, SIGTERM);
				std::_Exit(3);
			}
		}
	}
}

Channel &chan(int src, int dst) { return g_sh->chan[src * g_size + dst]; }

void send_chunk(Channel &c, const char *p, size_t n) {
	std::memcpy(c.data, p, n);
	c.len = n;
	c.full.store(1, std::memory_order_release);
}

size_t recv_chunk(Channel &c, char *p, size_t cap) {
	size_t n = c.len < cap ? c.len : cap;
	std::memcpy(p, c.data, n);
	c.full.store(0, std::memory_order_release);
	return n;
}

void check_size(size_t bytes, const char *what) {
	if (bytes > kSlot) {
		std::fprintf(stderr, "mpi_shm: %s payload of %zu bytes exceeds the %zu-byte slot\n", what, bytes, kSlot);
		std::abort();
	}
}

template<typename T>
void sum_slots(void *r, int n) {
	T *out = static_cast<T *>(r);
	for (int i = 0; i < n; i++) {
		T s = reinterpret_cast<const T *>(g_sh->slot[0])[i];
		for (int k = 1; k < g_size; k++) s += reinterpret_cast<const T *>(g_sh->slot[k])[i];
		out[i] = s;
	}
}

void reduce_into(void *r, int n, MPI_Datatype t) {
	if (t == MPI_INT) sum_slots<int>(r, n);
	else sum_slots<double>(r, n);
}

}// namespace

extern "C" {

int MPI_Init(int *, char ***) {
	const char *env = std::getenv("E3D_MPI_RANKS");
	g_size = env ? std::atoi(env) : 1;
	if (g_size < 1 || g_size > kMaxRanks) {
		std::fprintf(stderr, "mpi_shm: E3D_MPI_RANKS must be 1..%d\n", kMaxRanks);
		std::exit(2);
	}
	if (const char *t = std::getenv("E3D_MPI_TIMEOUT")) g_timeout = std::atof(t);
	const size_t bytes = sizeof(Shared) + ((size_t) g_size * g_size - 1) * sizeof(Channel);
	void *p = mmap(nullptr, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
	if (p == MAP_FAILED) {
		std::perror("mpi_shm: mmap");
		std::exit(2);
	}
	g_sh = static_cast<Shared *>(p);// zero-filled by mmap
	// the ranks form their own process group, so that a rank that gives up stops only them
	if (g_size > 1) setpgid(0, 0);
	std::fflush(nullptr);
	for (int r = 1; r < g_size; r++) {
		pid_t pid = fork();
		if (pid < 0) {
			std::perror("mpi_shm: fork");
			std::exit(2);
		}
		if (pid == 0) {
			g_rank = r;
			g_children.clear();
			return MPI_SUCCESS;
		}
		g_children.push_back(pid);
	}
	return MPI_SUCCESS;
}

int MPI_Finalize(void) {
	MPI_Barrier(MPI_COMM_WORLD);
	if (g_rank == 0) {
		int status = 0;
		for (pid_t c : g_children) waitpid(c, &status, 0);
	}
	return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm, int *rank) {
	*rank = g_rank;
	return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm, int *size) {
	*size = g_size;
	return MPI_SUCCESS;
}

double MPI_Wtime(void) { return now(); }

int MPI_Barrier(MPI_Comm) {
	if (g_size == 1) return MPI_SUCCESS;
	const int phase = g_phase;
	g_phase ^= 1;
	if (g_sh->bar_count.fetch_add(1) == g_size - 1) {
		g_sh->bar_count.store(0);
		g_sh->bar_phase.store(phase ^ 1);
	} else {
		wait_until([&] { return g_sh->bar_phase.load() != phase; }, "MPI_Barrier");
	}
	return MPI_SUCCESS;
}

int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm c) {
	const size_t bytes = (size_t) n * (size_t) t;
	check_size(bytes, "MPI_Allreduce");
	std::memcpy(g_sh->slot[g_rank], s, bytes);
	MPI_Barrier(c);
	reduce_into(r, n, t);
	MPI_Barrier(c);
	return MPI_SUCCESS;
}

int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int root, MPI_Comm c) {
	const size_t bytes = (size_t) n * (size_t) t;
	check_size(bytes, "MPI_Reduce");
	std::memcpy(g_sh->slot[g_rank], s, bytes);
	MPI_Barrier(c);
	if (g_rank == root) reduce_into(r, n, t);
	MPI_Barrier(c);
	return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm c) {
	const size_t bytes = (size_t) n * (size_t) t;
	check_size(bytes, "MPI_Bcast");
	if (g_rank == root) std::memcpy(g_sh->slot[root], buf, bytes);
	MPI_Barrier(c);
	if (g_rank != root) std::memcpy(buf, g_sh->slot[root], bytes);
	MPI_Barrier(c);
	return MPI_SUCCESS;
}

int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int root, MPI_Comm c) {
	const size_t bytes = (size_t) n * (size_t) t;
	check_size(bytes, "MPI_Gather");
	std::memcpy(g_sh->slot[g_rank], s, bytes);
	MPI_Barrier(c);
	if (g_rank == root)
		for (int k = 0; k < g_size; k++) std::memcpy(static_cast<char *>(r) + k * bytes, g_sh->slot[k], bytes);
	MPI_Barrier(c);
	return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int n, MPI_Datatype t, int dest, int, MPI_Comm) {
	Channel &c = chan(g_rank, dest);
	const char *p = static_cast<const char *>(buf);
	size_t left = (size_t) n * (size_t) t;
	do {
		wait_until([&] { return c.full.load(std::memory_order_acquire) == 0; }, "MPI_Send");
		const size_t k = left < kChunk ? left : kChunk;
		send_chunk(c, p, k);
		p += k;
		left -= k;
	} while (left > 0);
	return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int n, MPI_Datatype t, int src, int, MPI_Comm, MPI_Status *) {
	Channel &c = chan(src, g_rank);
	char *p = static_cast<char *>(buf);
	size_t left = (size_t) n * (size_t) t;
	do {
		wait_until([&] { return c.full.load(std::memory_order_acquire) == 1; }, "MPI_Recv");
		const size_t k = recv_chunk(c, p, left);
		p += k;
		left -= k;
	} while (left > 0);
	return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sbuf, int sn, MPI_Datatype st, int dest, int, void *rbuf, int rn, MPI_Datatype rt,
                 int src, int, MPI_Comm, MPI_Status *) {
	Channel &out = chan(g_rank, dest);
	Channel &in = chan(src, g_rank);
	const char *sp = static_cast<const char *>(sbuf);
	char *rp = static_cast<char *>(rbuf);
	size_t sleft = (size_t) sn * (size_t) st, rleft = (size_t) rn * (size_t) rt;
	bool sent_any = false, got_any = false;  // zero-byte messages still pass one (empty) chunk
	while (!(sent_any && sleft == 0) || !(got_any && rleft == 0)) {
		bool progressed = false;
		if (!(sent_any && sleft == 0) && out.full.load(std::memory_order_acquire) == 0) {
			const size_t k = sleft < kChunk ? sleft : kChunk;
			send_chunk(out, sp, k);
			sp += k;
			sleft -= k;
			sent_any = progressed = true;
		}
		if (!(got_any && rleft == 0) && in.full.load(std::memory_order_acquire) == 1) {
			const size_t k = recv_chunk(in, rp, rleft);
			rp += k;
			rleft -= k;
			got_any = progressed = true;
		}
		if (!progressed)
			wait_until([&] {
				return (!(sent_any && sleft == 0) && out.full.load(std::memory_order_acquire) == 0) ||
				       (!(got_any && rleft == 0) && in.full.load(std::memory_order_acquire) == 1);
			}, "MPI_Sendrecv");
	}
	return MPI_SUCCESS;
}

}// extern "C"
