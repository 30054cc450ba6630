/* The seam's device-matrix cache and settings (see KPMSeamB200.h). */
#include "KPMSeamB200.h"

#include "TBTK/HoppingAmplitudeSet.h"
#include "TBTK/Streams.h"
#include "TBTK/TBTKMacros.h"

#include <cstdlib>
#include <cstring>
#include <list>
#include <mutex>
#include <string>
#include <vector>

using namespace std;

namespace TBTK{
namespace B200{

namespace{

const unsigned int kCacheSize = 4;

/* 64-bit mixing of one word into a running hash (splitmix64 finaliser). */
inline uint64_t mix(uint64_t h, uint64_t v){
	uint64_t z = h ^ (v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2));
	z = (z ^ (z >> 30))*0xbf58476d1ce4e5b9ull;
	z = (z ^ (z >> 27))*0x94d049bb133111ebull;
	return z ^ (z >> 31);
}

inline uint64_t mixIndex(uint64_t h, const Index &index){
	h = mix(h, index.getSize());
	for(unsigned int n = 0; n < index.getSize(); n++)
		h = mix(h, (uint64_t)(int64_t)(int)index.at(n));
	return h;
}

inline uint64_t bits(double d){
	uint64_t u;
	memcpy(&u, &d, sizeof(u));
	return u;
}

/* Hash of every amplitude of the set with its to and from indices, in the
 * set's iteration order, and the number of amplitudes. */
uint64_t fingerprint(const HoppingAmplitudeSet &set, uint64_t *count){
	uint64_t h = 0x243f6a8885a308d3ull, n = 0;
	for(
		HoppingAmplitudeSet::ConstIterator it = set.cbegin();
		it != set.cend();
		++it
	){
		const HoppingAmplitude &ha = *it;
		const complex<double> a = ha.getAmplitude();
		h = mixIndex(mixIndex(h, ha.getToIndex()), ha.getFromIndex());
		h = mix(mix(h, bits(a.real())), bits(a.imag()));
		n++;
	}
	*count = n;
	return h;
}

struct Entry{
	const Model *model;
	double scaleFactor;
	int device;
	uint64_t hash, count;
	shared_ptr<tbtkkpm_matrix> matrix;
};

mutex cacheLock;
/* Most recently used first.  Allocated once and never freed: device
 * handles must not be destroyed after the CUDA runtime has shut down. */
list<Entry> &cache(){
	static list<Entry> *entries = new list<Entry>();
	return *entries;
}

shared_ptr<tbtkkpm_matrix> build(
	const HoppingAmplitudeSet &set,
	double scaleFactor,
	const char *where
){
	vector<uint32_t> rows, cols;
	vector<double> values;
	for(
		HoppingAmplitudeSet::ConstIterator it = set.cbegin();
		it != set.cend();
		++it
	){
		const HoppingAmplitude &ha = *it;
		const complex<double> a = ha.getAmplitude();
		rows.push_back(set.getBasisIndex(ha.getToIndex()));
		cols.push_back(set.getBasisIndex(ha.getFromIndex()));
		values.push_back(a.real());
		values.push_back(a.imag());
	}
	tbtkkpm_matrix *m = nullptr;
	check(
		tbtkkpm_matrix_create_triplets(
			rows.data(),
			cols.data(),
			values.data(),
			rows.size(),
			set.getBasisSize(),
			scaleFactor,
			&m
		),
		where
	);
	const uint32_t width = batchWidth();
	if(width != 0){
		check(
			tbtkkpm_matrix_set_batch_width(m, TBTKKPM_MIXED, width),
			where
		);
		if(width <= 128){
			check(
				tbtkkpm_matrix_set_batch_width(
					m,
					TBTKKPM_FP64,
					width
				),
				where
			);
		}
	}
	return shared_ptr<tbtkkpm_matrix>(m, tbtkkpm_matrix_destroy);
}

};	//End of anonymous namespace

void check(int status, const char *where){
	if(status != TBTKKPM_OK){
		TBTKExit(where, tbtkkpm_last_error(), "");
	}
}

int precision(){
	const char *p = getenv("TBTK_B200_PRECISION");
	if(p == nullptr || strcmp(p, "fp64") == 0 || p[0] == '\0')
		return TBTKKPM_FP64;
	if(strcmp(p, "mixed") == 0)
		return TBTKKPM_MIXED;
	TBTKExit(
		"TBTK_B200_PRECISION",
		"Unknown precision '" << p << "'.",
		"Use fp64 or mixed."
	);
	return TBTKKPM_FP64;
}

uint32_t batchWidth(){
	const char *p = getenv("TBTK_B200_BATCH");
	if(p == nullptr || p[0] == '\0')
		return 0;
	char *end = nullptr;
	const long v = strtol(p, &end, 10);
	TBTKAssert(
		end != p && *end == '\0' && v >= 0 && v <= 256,
		"TBTK_B200_BATCH",
		"Expected a batch width in [0, 256], got '" << p << "'.",
		""
	);
	return (uint32_t)v;
}

shared_ptr<tbtkkpm_matrix> deviceMatrix(
	const Model &model,
	double scaleFactor,
	int device,
	const char *where
){
	const HoppingAmplitudeSet &set = model.getHoppingAmplitudeSet();
	uint64_t count = 0;
	const uint64_t hash = fingerprint(set, &count);
	lock_guard<mutex> lock(cacheLock);
	list<Entry> &entries = cache();
	for(list<Entry>::iterator it = entries.begin(); it != entries.end(); ++it){
		if(
			it->model == &model
			&& it->scaleFactor == scaleFactor
			&& it->device == device
		){
			if(it->hash == hash && it->count == count){
				entries.splice(entries.begin(), entries, it);
				return entries.front().matrix;
			}
			entries.erase(it);
			break;
		}
	}
	Entry e;
	e.model = &model;
	e.scaleFactor = scaleFactor;
	e.device = device;
	e.hash = hash;
	e.count = count;
	e.matrix = build(set, scaleFactor, where);
	entries.push_front(e);
	while(entries.size() > kCacheSize)
		entries.pop_back();
	return entries.front().matrix;
}

};	//End of namespace B200
};	//End of namespace TBTK
