// Judy-API shim implementation (oracle / test infrastructure only).
//
// Every Judy array handle is a pointer to a heap object derived from JArr;
// a NULL handle is an empty array, as in libJudy.  The free calls accept a
// handle of any kind (the reference frees a JudySL array with JHSFA in
// common/mapint.h:105), so destruction goes through a virtual destructor.
#include "Judy.h"

#include <cstring>
#include <map>
#include <set>
#include <string>

namespace {

struct JArr {
	virtual ~JArr() {}
	virtual Word_t bytes() const = 0;
};

struct JL : JArr {
	std::map<Word_t, Word_t> m;
	// maximal runs of consecutive keys, start -> last key, so that
	// JudyLFirstEmpty answers in O(log n) as Judy's does (a linear scan made
	// the reference's Map::set, and so mesh building, quadratic)
	std::map<Word_t, Word_t> runs;
	Word_t bytes() const { return m.size() * 48; }
	void run_insert(Word_t k) {
		std::map<Word_t, Word_t>::iterator nx = runs.upper_bound(k);
		bool join_prev = false;
		std::map<Word_t, Word_t>::iterator pv = nx;
		if (pv != runs.begin()) {
			--pv;
			if (pv->second != ~0UL && pv->second + 1 == k) join_prev = true;
		}
		bool join_next = k != ~0UL && nx != runs.end() && nx->first == k + 1;
		if (join_prev && join_next) { pv->second = nx->second; runs.erase(nx); }
		else if (join_prev) pv->second = k;
		else if (join_next) { Word_t last = nx->second; runs.erase(nx); runs[k] = last; }
		else runs[k] = k;
	}
	void run_erase(Word_t k) {
		std::map<Word_t, Word_t>::iterator r = runs.upper_bound(k);
		--r;                                     // the run holding k
		Word_t a = r->first, b = r->second;
		runs.erase(r);
		if (a < k) runs[a] = k - 1;
		if (k < b) runs[k + 1] = b;
	}
};

struct J1 : JArr {
	std::set<Word_t> s;
	Word_t bytes() const { return s.size() * 40; }
};

struct JStr : JArr {       // JudyHS and JudySL: byte-string keys
	std::map<std::string, Word_t> m;
	Word_t bytes() const { return m.size() * 64; }
};

template <class T>
T *get(Pcvoid_t p) { return (T *) const_cast<void *>(p); }

template <class T>
T *get_or_make(PPvoid_t pp) {
	if (*pp == NULL) *pp = (Pvoid_t) new T();
	return (T *) *pp;
}

Word_t free_any(PPvoid_t pp) {
	if (pp == NULL || *pp == NULL) return 0;
	JArr *a = (JArr *) *pp;
	Word_t b = a->bytes();
	delete a;
	*pp = NULL;
	return b;
}

inline PPvoid_t slot(Word_t &v) { return (PPvoid_t) &v; }

} // namespace

// ---------------------------------------------------------------- JudyL

PPvoid_t JudyLIns(PPvoid_t PPArray, Word_t Index, PJError_t) {
	JL *a = get_or_make<JL>(PPArray);
	std::map<Word_t, Word_t>::iterator it = a->m.lower_bound(Index);
	if (it == a->m.end() || it->first != Index) {
		it = a->m.insert(it, std::make_pair(Index, (Word_t) 0));   // value-initialised to 0 when new
		a->run_insert(Index);
	}
	return slot(it->second);
}

int JudyLDel(PPvoid_t PPArray, Word_t Index, PJError_t) {
	if (*PPArray == NULL) return 0;
	JL *a = get<JL>(*PPArray);
	int rc = (int) a->m.erase(Index);
	if (rc) a->run_erase(Index);
	if (a->m.empty()) free_any(PPArray);
	return rc;
}

PPvoid_t JudyLGet(Pcvoid_t PArray, Word_t Index, PJError_t) {
	if (PArray == NULL) return NULL;
	JL *a = get<JL>(PArray);
	std::map<Word_t, Word_t>::iterator it = a->m.find(Index);
	return it == a->m.end() ? NULL : slot(it->second);
}

Word_t JudyLCount(Pcvoid_t PArray, Word_t I1, Word_t I2, PJError_t) {
	if (PArray == NULL || I1 > I2) return 0;
	JL *a = get<JL>(PArray);
	// whole-range counts (Array::count(), once per add_vertex / add_hex) in
	// constant time, as Judy's population counters give them
	if (a->m.empty()) return 0;
	if (I1 <= a->m.begin()->first && I2 >= a->m.rbegin()->first) return (Word_t) a->m.size();
	Word_t n = 0;
	for (std::map<Word_t, Word_t>::iterator it = a->m.lower_bound(I1); it != a->m.end() && it->first <= I2; ++it) n++;
	return n;
}

PPvoid_t JudyLByCount(Pcvoid_t PArray, Word_t Count, Word_t *PIndex, PJError_t) {
	if (PArray == NULL || Count == 0) return NULL;
	JL *a = get<JL>(PArray);
	if (Count > a->m.size()) return NULL;
	std::map<Word_t, Word_t>::iterator it = a->m.begin();
	for (Word_t k = 1; k < Count; k++) ++it;
	*PIndex = it->first;
	return slot(it->second);
}

Word_t JudyLFreeArray(PPvoid_t PPArray, PJError_t) { return free_any(PPArray); }

Word_t JudyLMemUsed(Pcvoid_t PArray) { return PArray ? ((JArr *) PArray)->bytes() : 0; }

PPvoid_t JudyLFirst(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return NULL;
	JL *a = get<JL>(PArray);
	std::map<Word_t, Word_t>::iterator it = a->m.lower_bound(*PIndex);
	if (it == a->m.end()) return NULL;
	*PIndex = it->first;
	return slot(it->second);
}

PPvoid_t JudyLNext(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return NULL;
	JL *a = get<JL>(PArray);
	std::map<Word_t, Word_t>::iterator it = a->m.upper_bound(*PIndex);
	if (it == a->m.end()) return NULL;
	*PIndex = it->first;
	return slot(it->second);
}

PPvoid_t JudyLLast(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return NULL;
	JL *a = get<JL>(PArray);
	std::map<Word_t, Word_t>::iterator it = a->m.upper_bound(*PIndex);
	if (it == a->m.begin()) return NULL;
	--it;
	*PIndex = it->first;
	return slot(it->second);
}

PPvoid_t JudyLPrev(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return NULL;
	JL *a = get<JL>(PArray);
	std::map<Word_t, Word_t>::iterator it = a->m.lower_bound(*PIndex);
	if (it == a->m.begin()) return NULL;
	--it;
	*PIndex = it->first;
	return slot(it->second);
}

int JudyLFirstEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	Word_t i = *PIndex;
	if (PArray == NULL) return 1;
	JL *a = get<JL>(PArray);
	std::map<Word_t, Word_t>::iterator r = a->runs.upper_bound(i);
	if (r != a->runs.begin()) {
		--r;
		if (r->second >= i) {                    // i is taken: the slot after its run
			if (r->second == ~0UL) return 0;
			i = r->second + 1;
		}
	}
	*PIndex = i;
	return 1;
}

// ---------------------------------------------------------------- Judy1

int Judy1Set(PPvoid_t PPArray, Word_t Index, PJError_t) {
	return get_or_make<J1>(PPArray)->s.insert(Index).second ? 1 : 0;
}

int Judy1Unset(PPvoid_t PPArray, Word_t Index, PJError_t) {
	if (*PPArray == NULL) return 0;
	J1 *a = get<J1>(*PPArray);
	int rc = (int) a->s.erase(Index);
	if (a->s.empty()) free_any(PPArray);
	return rc;
}

int Judy1Test(Pcvoid_t PArray, Word_t Index, PJError_t) {
	return PArray != NULL && get<J1>(PArray)->s.count(Index) ? 1 : 0;
}

Word_t Judy1Count(Pcvoid_t PArray, Word_t I1, Word_t I2, PJError_t) {
	if (PArray == NULL || I1 > I2) return 0;
	J1 *a = get<J1>(PArray);
	if (a->s.empty()) return 0;
	if (I1 <= *a->s.begin() && I2 >= *a->s.rbegin()) return (Word_t) a->s.size();
	Word_t n = 0;
	for (std::set<Word_t>::iterator it = a->s.lower_bound(I1); it != a->s.end() && *it <= I2; ++it) n++;
	return n;
}

int Judy1ByCount(Pcvoid_t PArray, Word_t Count, Word_t *PIndex, PJError_t) {
	if (PArray == NULL || Count == 0) return 0;
	J1 *a = get<J1>(PArray);
	if (Count > a->s.size()) return 0;
	std::set<Word_t>::iterator it = a->s.begin();
	for (Word_t k = 1; k < Count; k++) ++it;
	*PIndex = *it;
	return 1;
}

Word_t Judy1FreeArray(PPvoid_t PPArray, PJError_t) { return free_any(PPArray); }

int Judy1First(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return 0;
	J1 *a = get<J1>(PArray);
	std::set<Word_t>::iterator it = a->s.lower_bound(*PIndex);
	if (it == a->s.end()) return 0;
	*PIndex = *it;
	return 1;
}

int Judy1Next(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return 0;
	J1 *a = get<J1>(PArray);
	std::set<Word_t>::iterator it = a->s.upper_bound(*PIndex);
	if (it == a->s.end()) return 0;
	*PIndex = *it;
	return 1;
}

int Judy1Last(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return 0;
	J1 *a = get<J1>(PArray);
	std::set<Word_t>::iterator it = a->s.upper_bound(*PIndex);
	if (it == a->s.begin()) return 0;
	--it;
	*PIndex = *it;
	return 1;
}

int Judy1Prev(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (PArray == NULL) return 0;
	J1 *a = get<J1>(PArray);
	std::set<Word_t>::iterator it = a->s.lower_bound(*PIndex);
	if (it == a->s.begin()) return 0;
	--it;
	*PIndex = *it;
	return 1;
}

static bool j1_has(Pcvoid_t PArray, Word_t i) {
	return PArray != NULL && get<J1>(PArray)->s.count(i);
}

int Judy1FirstEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	Word_t i = *PIndex;
	while (j1_has(PArray, i)) {
		if (i == ~0UL) return 0;
		++i;
	}
	*PIndex = i;
	return 1;
}

int Judy1NextEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (*PIndex == ~0UL) return 0;
	Word_t i = *PIndex + 1;
	while (j1_has(PArray, i)) {
		if (i == ~0UL) return 0;
		++i;
	}
	*PIndex = i;
	return 1;
}

int Judy1LastEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	Word_t i = *PIndex;
	while (j1_has(PArray, i)) {
		if (i == 0) return 0;
		--i;
	}
	*PIndex = i;
	return 1;
}

int Judy1PrevEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t) {
	if (*PIndex == 0) return 0;
	Word_t i = *PIndex - 1;
	while (j1_has(PArray, i)) {
		if (i == 0) return 0;
		--i;
	}
	*PIndex = i;
	return 1;
}

// ---------------------------------------------------------------- JudyHS

PPvoid_t JudyHSIns(PPvoid_t PPArray, const void *Index, Word_t Length, PJError_t) {
	JStr *a = get_or_make<JStr>(PPArray);
	return slot(a->m[std::string((const char *) Index, Length)]);
}

PPvoid_t JudyHSGet(Pcvoid_t PArray, const void *Index, Word_t Length) {
	if (PArray == NULL) return NULL;
	JStr *a = get<JStr>(PArray);
	std::map<std::string, Word_t>::iterator it = a->m.find(std::string((const char *) Index, Length));
	return it == a->m.end() ? NULL : slot(it->second);
}

int JudyHSDel(PPvoid_t PPArray, const void *Index, Word_t Length, PJError_t) {
	if (*PPArray == NULL) return 0;
	JStr *a = get<JStr>(*PPArray);
	int rc = (int) a->m.erase(std::string((const char *) Index, Length));
	if (a->m.empty()) free_any(PPArray);
	return rc;
}

Word_t JudyHSFreeArray(PPvoid_t PPArray, PJError_t) { return free_any(PPArray); }

// ---------------------------------------------------------------- JudySL

PPvoid_t JudySLIns(PPvoid_t PPArray, const uint8_t *Index, PJError_t) {
	JStr *a = get_or_make<JStr>(PPArray);
	return slot(a->m[std::string((const char *) Index)]);
}

PPvoid_t JudySLGet(Pcvoid_t PArray, const uint8_t *Index, PJError_t) {
	if (PArray == NULL) return NULL;
	JStr *a = get<JStr>(PArray);
	std::map<std::string, Word_t>::iterator it = a->m.find(std::string((const char *) Index));
	return it == a->m.end() ? NULL : slot(it->second);
}

int JudySLDel(PPvoid_t PPArray, const uint8_t *Index, PJError_t) {
	if (*PPArray == NULL) return 0;
	JStr *a = get<JStr>(*PPArray);
	int rc = (int) a->m.erase(std::string((const char *) Index));
	if (a->m.empty()) free_any(PPArray);
	return rc;
}

PPvoid_t JudySLFirst(Pcvoid_t PArray, uint8_t *Index, PJError_t) {
	if (PArray == NULL) return NULL;
	JStr *a = get<JStr>(PArray);
	std::map<std::string, Word_t>::iterator it = a->m.lower_bound(std::string((const char *) Index));
	if (it == a->m.end()) return NULL;
	std::strcpy((char *) Index, it->first.c_str());
	return slot(it->second);
}

Word_t JudySLFreeArray(PPvoid_t PPArray, PJError_t) { return free_any(PPArray); }
