/* Stand-in for the reference's CPUTree.h, which its main.h includes
 * (main.h:22) but the repository does not contain.  Nothing on the hot path
 * uses it. */
#ifndef CPUTREE_H
#define CPUTREE_H
#endif
