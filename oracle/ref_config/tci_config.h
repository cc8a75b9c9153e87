/* Hand-written TCI threading configuration: pthreads threads, pthread
 * spinlock, spin barrier (what the reference's configure picks for
 * --enable-threading=pthreads on Linux). */
#ifndef _TCI_CONFIG_H_
#define _TCI_CONFIG_H_
#define TCI_USE_ATOMIC_SPINLOCK  0
#define TCI_USE_OMP_LOCK         0
#define TCI_USE_OPENMP_THREADS   0
#define TCI_USE_WINDOWS_THREADS  0
#define TCI_USE_TBB_THREADS      0
#define TCI_USE_PPL_THREADS      0
#define TCI_USE_OMPTASK_THREADS  0
#define TCI_USE_DISPATCH_THREADS 0
#define TCI_USE_OSX_SPINLOCK     0
#define TCI_USE_OS_UNFAIR_LOCK   0
#define TCI_USE_PTHREADS_THREADS 1
#define TCI_USE_PTHREAD_BARRIER  0
#define TCI_USE_PTHREAD_MUTEX    0
#define TCI_USE_PTHREAD_SPINLOCK 1
#define TCI_USE_SPIN_BARRIER     1
#endif
