#pragma once
#include "carbon.h"
struct CEvent;
struct CMulticastTimeEvent;
typedef HRESULT (*CEventHandler)(CEvent *);
CMulticastTimeEvent *CMulticastTimeEvent_New();
HRESULT CMulticastTimeEvent_Invoke(CMulticastTimeEvent *, double time);
struct CTimeEvent : PyObject {};
