/*
 * Judy-API shim for building the Hermes3D reference as a test oracle.
 *
 * ORACLE / TEST INFRASTRUCTURE ONLY.  libJudy is not installed on this
 * machine; the reference's containers (common/array.h, arrayptr.h,
 * bitarray.h, map.h, maphs.h, mapord.h, mapint.h, freqmap.h) and a few
 * direct calls (src/precalc.cc:54-207, src/function.cc:139-159,
 * src/refmap.cc:779-792, src/function.h:170,326) use the Judy C API.
 * This header re-implements the documented semantics of that API on top of
 * the C++ standard library:
 *
 *   JudyL  : ordered map  Word_t -> Word_t value slot   (JL* macros)
 *   Judy1  : ordered set of Word_t                       (J1* macros)
 *   JudyHS : map  byte-string -> Word_t value slot       (JHS* macros)
 *   JudySL : ordered map  C string -> Word_t value slot  (JSL* macros)
 *
 * Ordered iteration (First/Next/Last/Prev) follows ascending index order,
 * which is what drives the reference's FOR_ALL_* loops and therefore its
 * DOF numbering.  Value slots returned by the insert/get calls stay valid
 * until the index is deleted (std::map nodes are stable), a stronger
 * guarantee than libJudy gives, so every valid use of the real library is
 * also valid here.  No libJudy source was used; only its public manual
 * pages' description of each call.
 */
#ifndef H3D_ORACLE_JUDY_SHIM_H
#define H3D_ORACLE_JUDY_SHIM_H

#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

typedef unsigned long Word_t, *PWord_t;
typedef void *Pvoid_t, **PPvoid_t;
typedef const void *Pcvoid_t;

typedef struct J_UDY_ERROR_STRUCT {
	int je_Errno;
	int je_ErrID;
	Word_t je_reserved[4];
} JError_t, *PJError_t;

#define PJE0 ((PJError_t) 0)
#define PPJERR ((PPvoid_t) (~0UL))
#define PJERR ((Pvoid_t) (~0UL))
#define JERR (-1)

/* ---- JudyL ---- */
PPvoid_t JudyLIns(PPvoid_t PPArray, Word_t Index, PJError_t PJError);
int JudyLDel(PPvoid_t PPArray, Word_t Index, PJError_t PJError);
PPvoid_t JudyLGet(Pcvoid_t PArray, Word_t Index, PJError_t PJError);
Word_t JudyLCount(Pcvoid_t PArray, Word_t Index1, Word_t Index2, PJError_t PJError);
PPvoid_t JudyLByCount(Pcvoid_t PArray, Word_t Count, Word_t *PIndex, PJError_t PJError);
Word_t JudyLFreeArray(PPvoid_t PPArray, PJError_t PJError);
Word_t JudyLMemUsed(Pcvoid_t PArray);
PPvoid_t JudyLFirst(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
PPvoid_t JudyLNext(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
PPvoid_t JudyLLast(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
PPvoid_t JudyLPrev(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int JudyLFirstEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);

/* ---- Judy1 ---- */
int Judy1Set(PPvoid_t PPArray, Word_t Index, PJError_t PJError);
int Judy1Unset(PPvoid_t PPArray, Word_t Index, PJError_t PJError);
int Judy1Test(Pcvoid_t PArray, Word_t Index, PJError_t PJError);
Word_t Judy1Count(Pcvoid_t PArray, Word_t Index1, Word_t Index2, PJError_t PJError);
int Judy1ByCount(Pcvoid_t PArray, Word_t Count, Word_t *PIndex, PJError_t PJError);
Word_t Judy1FreeArray(PPvoid_t PPArray, PJError_t PJError);
int Judy1First(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1Next(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1Last(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1Prev(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1FirstEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1NextEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1LastEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);
int Judy1PrevEmpty(Pcvoid_t PArray, Word_t *PIndex, PJError_t PJError);

/* ---- JudyHS ---- */
PPvoid_t JudyHSIns(PPvoid_t PPArray, const void *Index, Word_t Length, PJError_t PJError);
PPvoid_t JudyHSGet(Pcvoid_t PArray, const void *Index, Word_t Length);
int JudyHSDel(PPvoid_t PPArray, const void *Index, Word_t Length, PJError_t PJError);
Word_t JudyHSFreeArray(PPvoid_t PPArray, PJError_t PJError);

/* ---- JudySL ---- */
PPvoid_t JudySLIns(PPvoid_t PPArray, const uint8_t *Index, PJError_t PJError);
PPvoid_t JudySLGet(Pcvoid_t PArray, const uint8_t *Index, PJError_t PJError);
int JudySLDel(PPvoid_t PPArray, const uint8_t *Index, PJError_t PJError);
PPvoid_t JudySLFirst(Pcvoid_t PArray, uint8_t *Index, PJError_t PJError);
Word_t JudySLFreeArray(PPvoid_t PPArray, PJError_t PJError);

/* The reference declares value pointers as `void *`; the Judy manual
 * declares them as PWord_t.  Assign through a cast so either compiles. */
#define J_ASSIGN_PV(PV, EXPR) ((PV) = (__typeof__(PV)) (EXPR))

#define JLI(PV, PA, I)        J_ASSIGN_PV(PV, JudyLIns(&(PA), (I), PJE0))
#define JLD(RC, PA, I)        ((RC) = JudyLDel(&(PA), (I), PJE0))
#define JLG(PV, PA, I)        J_ASSIGN_PV(PV, JudyLGet((PA), (I), PJE0))
#define JLC(RC, PA, I1, I2)   ((RC) = JudyLCount((PA), (I1), (I2), PJE0))
#define JLBC(PV, PA, N, I)    J_ASSIGN_PV(PV, JudyLByCount((PA), (N), &(I), PJE0))
#define JLFA(RC, PA)          ((RC) = JudyLFreeArray(&(PA), PJE0))
#define JLMU(RC, PA)          ((RC) = JudyLMemUsed(PA))
#define JLF(PV, PA, I)        J_ASSIGN_PV(PV, JudyLFirst((PA), &(I), PJE0))
#define JLN(PV, PA, I)        J_ASSIGN_PV(PV, JudyLNext((PA), &(I), PJE0))
#define JLL(PV, PA, I)        J_ASSIGN_PV(PV, JudyLLast((PA), &(I), PJE0))
#define JLP(PV, PA, I)        J_ASSIGN_PV(PV, JudyLPrev((PA), &(I), PJE0))
#define JLFE(RC, PA, I)       ((RC) = JudyLFirstEmpty((PA), &(I), PJE0))

#define J1S(RC, PA, I)        ((RC) = Judy1Set(&(PA), (I), PJE0))
#define J1U(RC, PA, I)        ((RC) = Judy1Unset(&(PA), (I), PJE0))
#define J1T(RC, PA, I)        ((RC) = Judy1Test((PA), (I), PJE0))
#define J1C(RC, PA, I1, I2)   ((RC) = Judy1Count((PA), (I1), (I2), PJE0))
#define J1BC(RC, PA, N, I)    ((RC) = Judy1ByCount((PA), (N), &(I), PJE0))
#define J1FA(RC, PA)          ((RC) = Judy1FreeArray(&(PA), PJE0))
#define J1F(RC, PA, I)        ((RC) = Judy1First((PA), &(I), PJE0))
#define J1N(RC, PA, I)        ((RC) = Judy1Next((PA), &(I), PJE0))
#define J1L(RC, PA, I)        ((RC) = Judy1Last((PA), &(I), PJE0))
#define J1P(RC, PA, I)        ((RC) = Judy1Prev((PA), &(I), PJE0))
#define J1FE(RC, PA, I)       ((RC) = Judy1FirstEmpty((PA), &(I), PJE0))
#define J1NE(RC, PA, I)       ((RC) = Judy1NextEmpty((PA), &(I), PJE0))
#define J1LE(RC, PA, I)       ((RC) = Judy1LastEmpty((PA), &(I), PJE0))
#define J1PE(RC, PA, I)       ((RC) = Judy1PrevEmpty((PA), &(I), PJE0))

#define JHSI(PV, PA, K, L)    J_ASSIGN_PV(PV, JudyHSIns(&(PA), (K), (L), PJE0))
#define JHSG(PV, PA, K, L)    J_ASSIGN_PV(PV, JudyHSGet((PA), (K), (L)))
#define JHSD(RC, PA, K, L)    ((RC) = JudyHSDel(&(PA), (K), (L), PJE0))
#define JHSFA(RC, PA)         ((RC) = JudyHSFreeArray(&(PA), PJE0))

#define JSLI(PV, PA, K)       J_ASSIGN_PV(PV, JudySLIns(&(PA), (K), PJE0))
#define JSLG(PV, PA, K)       J_ASSIGN_PV(PV, JudySLGet((PA), (K), PJE0))
#define JSLD(RC, PA, K)       ((RC) = JudySLDel(&(PA), (K), PJE0))
#define JSLF(PV, PA, K)       J_ASSIGN_PV(PV, JudySLFirst((PA), (K), PJE0))
#define JSLFA(RC, PA)         ((RC) = JudySLFreeArray(&(PA), PJE0))

#endif
