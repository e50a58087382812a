/* Helpers shared by the host layer's files; not exported from libqld_host.so. */
#ifndef QLD_HOST_INTERNAL_H
#define QLD_HOST_INTERNAL_H

#define QLD_INTERNAL __attribute__((visibility("hidden")))

/* Record a printf-style message for qld_host_last_error() and return `code`. */
QLD_INTERNAL int qld_host_fail(int code, const char *fmt, ...)
    __attribute__((format(printf, 2, 3)));
/* Run fn(arg) on `threads` threads (the caller's included) and join them. */
QLD_INTERNAL void qld_run_threads(void *(*fn)(void *), void *arg, int threads);

#endif
