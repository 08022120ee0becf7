// Host worker pool of libtsuner_b200.so (tsu::host_parallel): every index
// runs exactly once per call, over thousands of back-to-back calls, from
// several caller threads at once, and again in a forked child (which must
// build its own pool).  Exit status 0 = all checks passed.
#include <signal.h>
#include <sys/wait.h>
#include <unistd.h>

#include <atomic>
#include <cstdio>
#include <functional>
#include <thread>
#include <vector>

namespace tsu {
int host_threads();
void host_parallel(int n, const std::function<void(int)> &fn);
}  // namespace tsu

static bool sums(int calls, int n, int salt) {
    for (int c = 0; c < calls; c++) {
        std::vector<std::atomic<int>> hits(n);
        for (auto &h : hits) h.store(0);
        std::atomic<long long> total{0};
        tsu::host_parallel(n, [&](int i) {
            hits[i].fetch_add(1);
            total.fetch_add((long long)i * salt);
        });
        for (int i = 0; i < n; i++)
            if (hits[i].load() != 1) {
                fprintf(stderr, "call %d: index %d ran %d times\n", c, i, hits[i].load());
                return false;
            }
        if (total.load() != (long long)salt * n * (n - 1) / 2) {
            fprintf(stderr, "call %d: bad total\n", c);
            return false;
        }
    }
    return true;
}

int main() {
    alarm(120);  // a deadlock ends the program instead of the test run
    const int nt = tsu::host_threads();
    if (nt < 1) return 1;
    printf("threads %d\n", nt);
    if (!sums(3000, 7, 1) || !sums(200, 1000, 3) || !sums(500, 1, 5) || !sums(10, 0, 1)) return 2;
    std::vector<std::thread> callers;
    std::atomic<int> bad{0};
    for (int t = 0; t < 4; t++)
        callers.emplace_back([&, t] {
            if (!sums(400, 33 + t, t + 2)) bad.fetch_add(1);
        });
    for (auto &th : callers) th.join();
    if (bad.load()) return 3;
    pid_t pid = fork();
    if (pid == 0) {
        alarm(60);
        _exit(sums(300, 64, 7) ? 0 : 4);
    }
    int status = 0;
    if (waitpid(pid, &status, 0) != pid || !WIFEXITED(status) || WEXITSTATUS(status) != 0) return 5;
    if (!sums(300, 64, 9)) return 6;  // the parent's pool still works after the fork
    printf("ok\n");
    return 0;
}
