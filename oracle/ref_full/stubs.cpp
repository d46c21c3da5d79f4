// Stand-ins for the reference's TIFF and EER readers (libtiff is absent) and
// for CFullSpectrum::mEmbedCTF, whose source is commented out in the
// reference tree (FindCtf/CFullSpectrum.cpp:76-) and exists only in a
// shipped object file that is not used here.  The checker runs the reference
// on MRC movies with CTF estimation off (-Cs 0), which never reaches these.
#include "TiffUtil/CTiffFileInc.h"
#include "EerUtil/CEerUtilInc.h"
#include "FindCtf/CFindCtfInc.h"

using namespace MotionCor2;

TiffUtil::CLoadTiffHeader::CLoadTiffHeader(void) {}
TiffUtil::CLoadTiffHeader::~CLoadTiffHeader(void) {}
bool TiffUtil::CLoadTiffHeader::DoIt(int) { return false; }
int TiffUtil::CLoadTiffHeader::GetMode(void) { return -1; }
void TiffUtil::CLoadTiffHeader::GetSize(int* p, int n) { for (int i = 0; i < n; ++i) p[i] = 0; }
TiffUtil::CLoadTiffImage::CLoadTiffImage(void) {}
TiffUtil::CLoadTiffImage::~CLoadTiffImage(void) {}
bool TiffUtil::CLoadTiffImage::SetFile(int) { return false; }
void* TiffUtil::CLoadTiffImage::DoIt(int) { return 0L; }
bool TiffUtil::CLoadTiffImage::DoIt(int, void*) { return false; }
bool TiffUtil::CLoadTiffStack::OpenFile(int*) { return false; }
void TiffUtil::CLoadTiffStack::AsyncLoad(void) {}
void* TiffUtil::CLoadTiffStack::GetPackage(void) { return 0L; }
bool EerUtil::CLoadEerMain::OpenFile(int*) { return false; }
void EerUtil::CLoadEerMain::AsyncLoad(void) {}
void* EerUtil::CLoadEerMain::GetPackage(void) { return 0L; }
void FindCtf::CFullSpectrum::mEmbedCTF(void) {}
