/* ref_detail_mid.h -- TEST INFRASTRUCTURE: opens the class that receives the
 * streamed member functions (see ref_detail_prefix.h). */
struct RefDetail {
