/* bucket.h -- drop-in for the reference header (include/bucket.h:22-26). */
#ifndef SCG_DROPIN_BUCKET_H_
#define SCG_DROPIN_BUCKET_H_
#include <vector>
namespace SC {
typedef struct {
    int L = 0;
    std::vector<int> pid;
    std::vector<unsigned char> codes;
} Bucket;
}  // namespace SC
#endif
