// Device-vector globals of the reference's front end (operators.cu:45-47, cm.cu:79) that
// its generated parser's drivers release at exit (bison.y:440-459). They keep the
// reference's thrust types so that the parser links unchanged; this engine never fills
// them, so they stay empty and no device memory is involved.
#include <thrust/device_vector.h>

thrust::device_vector<unsigned char> scratch;
thrust::device_vector<long long int> rcol_dev;
thrust::device_vector<int> ranj;
